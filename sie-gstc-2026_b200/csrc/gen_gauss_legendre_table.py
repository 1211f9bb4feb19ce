"""Regenerate gauss_legendre_table.inc: Gauss-Legendre rules with 1-20 points
on [0, 1], nodes ascending, weights summing to 1.

The rules are the classical Gauss-Legendre rules (nodes the roots of P_n),
computed here with numpy.polynomial.legendre.leggauss (eigenvalues of the
Jacobi matrix refined by Newton steps) and mapped from [-1, 1] by
t = (x + 1) / 2, w = w / 2. The solver being replaced tabulates the same
rules on [0, 1] (src/sie_mom/quadrature/gauss_legendre_rule.cpp) and its
kernels round each node and weight to float
(src/sie_mom/solvers/pec_solver.cu:67-75, dielectric/dielectric_solver.cu:179-197);
tests/test_variants_oracle.py checks that the float-rounded values agree.

Usage (maintainers):
    python gen_gauss_legendre_table.py > gauss_legendre_table.inc
"""

import numpy as np


def main() -> None:
    print("// Generated by gen_gauss_legendre_table.py: Gauss-Legendre rules on [0, 1],")
    print("// n = 1..20 points, rule n at offset n (n - 1) / 2, nodes ascending.")
    nodes, weights = [], []
    for n in range(1, 21):
        x, w = np.polynomial.legendre.leggauss(n)
        nodes += list(0.5 * (x + 1.0))
        weights += list(0.5 * w)
    print("static const double kGaussLegendreNodes[210] = {")
    for v in nodes:
        print(f"    {float(v)!r},")
    print("};")
    print("static const double kGaussLegendreWeights[210] = {")
    for v in weights:
        print(f"    {float(v)!r},")
    print("};")


if __name__ == "__main__":
    main()
