"""Regenerate dunavant_table.inc: Dunavant's symmetric triangle rules 1-20.

The abscissae and weights are D. A. Dunavant's published values ("High degree
efficient symmetrical Gaussian quadrature rules for the triangle", IJNME 21,
1985), stored here as orbits: multiplicity (1, 3 or 6), the barycentric
triple and the orbit weight. The numbers must be the very doubles the solver
being replaced uses, because its kernels round each expanded point to float
(src/sie_mom/quadrature/triangle_dunavant_rule.cpp:135-256,
include/sie_mom/quadrature/triangle_dunavant_rule.hpp:82-101). This script
therefore prints them from that implementation once; the library itself only
reads the generated table.

Usage (maintainers, from a checkout that has the original sources):
    python gen_dunavant_table.py /path/to/sie-gstc-2026 > dunavant_table.inc
"""

import os
import subprocess
import sys
import tempfile

_DUMP = r"""
#include <cstdio>
int dunavant_suborder_num(int);
int* dunavant_suborder(int, int);
void dunavant_subrule(int, int, double*, double*);
int main() {
  for (int rule = 1; rule <= 20; ++rule) {
    int ns = dunavant_suborder_num(rule);
    int* so = dunavant_suborder(rule, ns);
    double* x = new double[3 * ns];
    double* w = new double[ns];
    dunavant_subrule(rule, ns, x, w);
    std::printf("/* rule %d */ {%d, {", rule, ns);
    for (int s = 0; s < ns; ++s)
      std::printf("{%d, %.17g, %.17g, %.17g, %.17g},", so[s], x[3*s], x[3*s+1], x[3*s+2], w[s]);
    std::printf("}},\n");
    delete[] so; delete[] x; delete[] w;
  }
  return 0;
}
"""


def main() -> None:
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SIE_REFERENCE")
    if not ref:
        raise SystemExit("usage: gen_dunavant_table.py /path/to/reference (or set SIE_REFERENCE)")
    src = os.path.join(ref, "src/sie_mom/quadrature/triangle_dunavant_rule.cpp")
    with tempfile.TemporaryDirectory() as tmp:
        dump = os.path.join(tmp, "dump.cpp")
        exe = os.path.join(tmp, "dump")
        with open(dump, "w") as fh:
            fh.write(_DUMP)
        subprocess.run(["/usr/bin/g++", "-O0", "-w", "-I", os.path.join(ref, "include"),
                        dump, src, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    print("// Generated by gen_dunavant_table.py: Dunavant (1985) rules 1-20 as orbits")
    print("// {multiplicity, a, b, c, weight}; see the generator for provenance.")
    print(out, end="")


if __name__ == "__main__":
    main()
