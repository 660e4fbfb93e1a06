"""Make the patched copy of the reference's enflo/src/fv.cc whose FV::run
time loop runs on the B200 through libdspw.so (include/dspw.h).

    python3 patch_fv_run.py <reference>/enflo/src/fv.cc <out>/fv.cc

The copy gets two textual includes, both of this project's own code:
dspw_driver_helpers.inc after the file's `using namespace std;` (descriptor
from Parameter, network file reader, status check), and dspw_time_loop.inc in
place of FV::run's time loop (enflo/src/fv.cc:1258-1313: from the "Solving"
message to the end of the while loop, before the final progress line).  The
two anchors must each be found exactly once, else nothing is written.  The
reference's sources stay untouched; oracle/Makefile compiles the copy with
the reference's other objects and main.cc into oracle/_ref/enflo_dspw.
"""
import sys


def patch(src: str) -> str:
    use = "using namespace std;"
    if src.count(use) < 1:
        raise SystemExit("patch_fv_run: no 'using namespace std;' in fv.cc")
    i = src.index(use) + len(use)
    src = src[:i] + '\n#include "dspw_driver_helpers.inc"\n' + src[i:]
    start_anchor = '---Solving ...'
    if src.count(start_anchor) != 1:
        raise SystemExit("patch_fv_run: the loop's start anchor is not unique")
    s = src.rindex("\n", 0, src.index(start_anchor)) + 1          # start of that line
    end_anchor = "<<++t_percent<<"
    if src.count(end_anchor) != 1:
        raise SystemExit("patch_fv_run: the loop's end anchor is not unique")
    e = src.rindex("if(!disp_log)", s, src.index(end_anchor))      # the final progress line's test
    e = src.rindex("\n", 0, e) + 1
    return src[:s] + '#include "dspw_time_loop.inc"\n' + src[e:]


if __name__ == "__main__":
    text = open(sys.argv[1]).read()
    out = patch(text)
    with open(sys.argv[2], "w") as f:
        f.write(out)
