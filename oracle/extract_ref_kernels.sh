#!/bin/sh
# TEST INFRASTRUCTURE.  Writes a C++ file holding gsbn's own CPU kernels of the
# ProcUpdLazy path, cut by line range out of the gsbn sources where they lie,
# so that the oracle can run the reference's arithmetic itself (math mode
# MATH_REF).  The output goes to oracle/_ref/, which is git-ignored: nothing of
# the reference is committed.
#
#   src/gsbn/procedures/ProcUpdLazy/Proj.cpp:209-536
#       update_all_kernel_cpu, update_jxx_kernel_cpu,
#       update_row_kernel_cpu, update_col_kernel_cpu
#   src/gsbn/procedures/ProcUpdLazy/Pop.cpp:229-323
#       update_sup_kernel_1_cpu, update_sup_kernel_2_cpu,
#       update_sup_kernel_3_cpu
#
# These are free functions over raw pointers; they need only the standard
# headers that gsbn's Common.hpp includes and its `using namespace std`
# (include/gsbn/Common.hpp:4-34), so that exp/log on a float resolve to the
# float overloads exactly as in the gsbn build.  The line ranges are checked
# against the function heads before anything is written.
#
# usage: extract_ref_kernels.sh <gsbn source root> <output .cpp>
set -eu
ROOT=$1
OUT=$2
PROJ=$ROOT/src/gsbn/procedures/ProcUpdLazy/Proj.cpp
POP=$ROOT/src/gsbn/procedures/ProcUpdLazy/Pop.cpp

expect() {  # file line text
  got=$(sed -n "$2p" "$1" | tr -d '\r')
  case "$got" in
    "$3"*) ;;
    *) echo "extract_ref_kernels: $1:$2 is '$got', expected '$3'" >&2; exit 1 ;;
  esac
}
expect "$PROJ" 209 "void update_all_kernel_cpu("
expect "$PROJ" 310 "void update_jxx_kernel_cpu("
expect "$PROJ" 365 "void update_row_kernel_cpu("
expect "$PROJ" 481 "void update_col_kernel_cpu("
expect "$PROJ" 536 "}"
expect "$PROJ" 538 "void Proj::update_all_cpu("
expect "$POP" 229 "void update_sup_kernel_1_cpu("
expect "$POP" 263 "void update_sup_kernel_2_cpu("
expect "$POP" 305 "void update_sup_kernel_3_cpu("
expect "$POP" 323 "}"
expect "$POP" 325 "void Pop::update_sup_cpu()"

mkdir -p "$(dirname "$OUT")"
{
  echo "// Generated by oracle/extract_ref_kernels.sh from the gsbn sources."
  echo "#include <iomanip>"
  echo "#include <string>"
  echo "#include <vector>"
  echo "#include <math.h>"
  echo "#include <stdint.h>"
  echo "using namespace std;"
  echo "namespace gsbn {"
  echo "namespace proc_upd_lazy {"
  echo "#line 209 \"src/gsbn/procedures/ProcUpdLazy/Proj.cpp\""
  sed -n '209,536p' "$PROJ"
  echo "#line 229 \"src/gsbn/procedures/ProcUpdLazy/Pop.cpp\""
  sed -n '229,323p' "$POP"
  echo "}  // namespace proc_upd_lazy"
  echo "}  // namespace gsbn"
} > "$OUT.tmp"
mv "$OUT.tmp" "$OUT"
