// expr.cc -- recursive-descent parser and tree evaluator for param.in
// expressions (see expr.h).  Precedence, lowest first: | ; & ; comparisons ;
// + - ; * / ; unary - ! ; ^ (right associative) ; calls and parentheses.
#include "expr.h"

#include <cctype>
#include <cmath>
#include <cstdlib>

namespace dspw_host {

struct Expr::Node {
  enum Kind { NUM, VAR, UNARY, BINARY, CALL } kind;
  double value = 0;
  int var = 0;                 // 0..3 = x y z t
  char op = 0;                 // unary: '-' '!' ; binary: + - * / ^ < > l(<=) g(>=) = n(!=) & |
  std::string fn;
  std::vector<std::shared_ptr<Node>> args;
};

namespace {

using NodeP = std::shared_ptr<Expr::Node>;

class Parser {
 public:
  Parser(const std::string& s, const std::map<std::string, double>& c) : s_(s), c_(c) {}

  NodeP parse() {
    NodeP n = parse_or();
    skip();
    if (p_ != s_.size()) fail("unexpected text");
    return n;
  }

 private:
  const std::string& s_;
  const std::map<std::string, double>& c_;
  size_t p_ = 0;

  [[noreturn]] void fail(const std::string& what) {
    throw std::runtime_error("expression '" + s_ + "': " + what + " at position " + std::to_string(p_));
  }
  void skip() {
    while (p_ < s_.size() && std::isspace((unsigned char)s_[p_])) ++p_;
  }
  bool eat(const char* tok) {
    skip();
    size_t n = std::char_traits<char>::length(tok);
    if (s_.compare(p_, n, tok) == 0) {
      p_ += n;
      return true;
    }
    return false;
  }
  static NodeP bin(char op, NodeP a, NodeP b) {
    auto n = std::make_shared<Expr::Node>();
    n->kind = Expr::Node::BINARY;
    n->op = op;
    n->args = {a, b};
    return n;
  }
  NodeP parse_or() {
    NodeP a = parse_and();
    while (eat("|")) a = bin('|', a, parse_and());
    return a;
  }
  NodeP parse_and() {
    NodeP a = parse_cmp();
    while (eat("&")) a = bin('&', a, parse_cmp());
    return a;
  }
  NodeP parse_cmp() {
    NodeP a = parse_add();
    for (;;) {
      if (eat("<=")) a = bin('l', a, parse_add());
      else if (eat(">=")) a = bin('g', a, parse_add());
      else if (eat("!=")) a = bin('n', a, parse_add());
      else if (eat("<")) a = bin('<', a, parse_add());
      else if (eat(">")) a = bin('>', a, parse_add());
      else if (eat("=")) a = bin('=', a, parse_add());
      else return a;
    }
  }
  NodeP parse_add() {
    NodeP a = parse_mul();
    for (;;) {
      if (eat("+")) a = bin('+', a, parse_mul());
      else if (eat("-")) a = bin('-', a, parse_mul());
      else return a;
    }
  }
  NodeP parse_mul() {
    NodeP a = parse_unary();
    for (;;) {
      if (eat("*")) a = bin('*', a, parse_unary());
      else if (eat("/")) a = bin('/', a, parse_unary());
      else return a;
    }
  }
  NodeP parse_unary() {
    if (eat("-")) {
      auto n = std::make_shared<Expr::Node>();
      n->kind = Expr::Node::UNARY;
      n->op = '-';
      n->args = {parse_unary()};
      return n;
    }
    if (eat("!")) {
      auto n = std::make_shared<Expr::Node>();
      n->kind = Expr::Node::UNARY;
      n->op = '!';
      n->args = {parse_unary()};
      return n;
    }
    return parse_pow();
  }
  NodeP parse_pow() {
    NodeP a = parse_atom();
    if (eat("^")) return bin('^', a, parse_unary());   // right associative
    return a;
  }
  NodeP parse_atom() {
    skip();
    if (p_ >= s_.size()) fail("unexpected end");
    char ch = s_[p_];
    if (ch == '(') {
      ++p_;
      NodeP n = parse_or();
      if (!eat(")")) fail("missing ')'");
      return n;
    }
    if (std::isdigit((unsigned char)ch) || ch == '.') {
      char* end = nullptr;
      double v = std::strtod(s_.c_str() + p_, &end);
      if (end == s_.c_str() + p_) fail("bad number");
      p_ = end - s_.c_str();
      auto n = std::make_shared<Expr::Node>();
      n->kind = Expr::Node::NUM;
      n->value = v;
      return n;
    }
    if (std::isalpha((unsigned char)ch) || ch == '_') {
      size_t b = p_;
      while (p_ < s_.size() && (std::isalnum((unsigned char)s_[p_]) || s_[p_] == '_')) ++p_;
      std::string id = s_.substr(b, p_ - b);
      if (eat("(")) {
        auto n = std::make_shared<Expr::Node>();
        n->kind = Expr::Node::CALL;
        n->fn = id;
        if (!eat(")")) {
          do n->args.push_back(parse_or());
          while (eat(","));
          if (!eat(")")) fail("missing ')' after arguments of " + id);
        }
        check_call(*n);
        return n;
      }
      auto n = std::make_shared<Expr::Node>();
      if (id == "x" || id == "y" || id == "z" || id == "t") {
        n->kind = Expr::Node::VAR;
        n->var = id == "x" ? 0 : (id == "y" ? 1 : (id == "z" ? 2 : 3));
        return n;
      }
      n->kind = Expr::Node::NUM;
      auto it = c_.find(id);
      if (it != c_.end()) n->value = it->second;
      else if (id == "pi") n->value = M_PI;
      else if (id == "e") n->value = M_E;
      else fail("unknown name '" + id + "'");
      return n;
    }
    fail(std::string("unexpected character '") + ch + "'");
  }
  void check_call(const Expr::Node& n) {
    static const std::map<std::string, int> arity = {
        {"sin", 1}, {"cos", 1}, {"tan", 1}, {"asin", 1}, {"acos", 1}, {"atan", 1}, {"sinh", 1},
        {"cosh", 1}, {"tanh", 1}, {"exp", 1}, {"log", 1}, {"log10", 1}, {"sqrt", 1}, {"abs", 1},
        {"floor", 1}, {"ceil", 1}, {"int", 1}, {"atan2", 2}, {"pow", 2}, {"min", 2}, {"max", 2}, {"if", 3}};
    auto it = arity.find(n.fn);
    if (it == arity.end()) fail("unknown function '" + n.fn + "'");
    if ((int)n.args.size() != it->second) fail("wrong number of arguments to " + n.fn);
  }
};

double ev(const Expr::Node& n, const double v[4]) {
  switch (n.kind) {
    case Expr::Node::NUM: return n.value;
    case Expr::Node::VAR: return v[n.var];
    case Expr::Node::UNARY: {
      double a = ev(*n.args[0], v);
      return n.op == '-' ? -a : (a == 0.0 ? 1.0 : 0.0);
    }
    case Expr::Node::BINARY: {
      double a = ev(*n.args[0], v), b = ev(*n.args[1], v);
      switch (n.op) {
        case '+': return a + b;
        case '-': return a - b;
        case '*': return a * b;
        case '/': return a / b;
        case '^': return std::pow(a, b);
        case '<': return a < b ? 1.0 : 0.0;
        case '>': return a > b ? 1.0 : 0.0;
        case 'l': return a <= b ? 1.0 : 0.0;
        case 'g': return a >= b ? 1.0 : 0.0;
        case '=': return a == b ? 1.0 : 0.0;
        case 'n': return a != b ? 1.0 : 0.0;
        case '&': return (a != 0.0 && b != 0.0) ? 1.0 : 0.0;
        case '|': return (a != 0.0 || b != 0.0) ? 1.0 : 0.0;
      }
      return 0.0;
    }
    case Expr::Node::CALL: {
      const std::string& f = n.fn;
      double a = ev(*n.args[0], v);
      if (f == "if") return a != 0.0 ? ev(*n.args[1], v) : ev(*n.args[2], v);
      if (n.args.size() == 2) {
        double b = ev(*n.args[1], v);
        if (f == "pow") return std::pow(a, b);
        if (f == "atan2") return std::atan2(a, b);
        if (f == "min") return a < b ? a : b;
        return a > b ? a : b;   // max
      }
      if (f == "sin") return std::sin(a);
      if (f == "cos") return std::cos(a);
      if (f == "tan") return std::tan(a);
      if (f == "asin") return std::asin(a);
      if (f == "acos") return std::acos(a);
      if (f == "atan") return std::atan(a);
      if (f == "sinh") return std::sinh(a);
      if (f == "cosh") return std::cosh(a);
      if (f == "tanh") return std::tanh(a);
      if (f == "exp") return std::exp(a);
      if (f == "log") return std::log(a);
      if (f == "log10") return std::log10(a);
      if (f == "sqrt") return std::sqrt(a);
      if (f == "abs") return std::fabs(a);
      if (f == "floor") return std::floor(a);
      if (f == "ceil") return std::ceil(a);
      return std::trunc(a);   // int
    }
  }
  return 0.0;
}

}  // namespace

Expr::Expr(const std::string& text, const std::map<std::string, double>& constants) : text_(text) {
  Parser p(text_, constants);
  root_ = p.parse();
}

double Expr::eval(double x, double y, double z, double t) const {
  const double v[4] = {x, y, z, t};
  return ev(*root_, v);
}

}  // namespace dspw_host
