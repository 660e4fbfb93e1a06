// expr.h -- arithmetic expressions of param.in initial conditions, exact
// solutions and domain limits.
//
// The reference evaluates these with the third-party fparser library
// (enflo/src/fparser.h, variables "x,y,z,t", constant pi plus the constants
// section).  This is a small evaluator of the subset the examples use, written
// for this project: numbers, the variables x y z t, named constants, + - * / ^,
// unary - and !, comparisons < <= > >= = != (value 1 or 0), & and |,
// parentheses, and the functions sin cos tan asin acos atan atan2 sinh cosh
// tanh exp log log10 sqrt abs pow min max floor ceil int if.
#pragma once
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace dspw_host {

class Expr {
 public:
  // throws std::runtime_error with the position on a syntax error
  Expr(const std::string& text, const std::map<std::string, double>& constants);
  double eval(double x, double y, double z, double t) const;
  const std::string& text() const { return text_; }

  struct Node;

 private:
  std::string text_;
  std::shared_ptr<Node> root_;
};

}  // namespace dspw_host
