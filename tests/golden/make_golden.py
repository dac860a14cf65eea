"""Regenerate the golden fixtures of this directory from the reference checkout.

Reads the reference's committed plane-wave reflectance tables
(``comparisons/gila_airy/results/{film,stack}.tsv``: columns pol, angle, R_tmm, R_own,
R_gila) and writes ``reflectance_{film,stack}.json`` with the film definitions of
``comparisons/gila_airy/airy_comparison.jl:26-29`` (χ, thickness in λ; vacuum on both
sides, λ = 1, ω = k0 = 2π). Run once where the reference is mounted:

    python tests/golden/make_golden.py /path/to/YellowThinFilms
"""
import json
import os
import sys

FILMS = {"film": [[1.25, 0.0, 0.5]], "stack": [[1.25, 0.0, 0.25], [3.0, 0.0, 0.1875], [1.0, 0.1, 0.125]]}


def main(root):
    here = os.path.dirname(os.path.abspath(__file__))
    for name, films in FILMS.items():
        path = os.path.join(root, "comparisons", "gila_airy", "results", f"{name}.tsv")
        rows = [l.split("\t") for l in open(path).read().strip().split("\n")[1:]]
        out = dict(source=f"comparisons/gila_airy/results/{name}.tsv", films_chi_re_im_d=films,
                   rows=[dict(pol=p, angle=float(a), R_tmm=float(t), R_own=float(o)) for p, a, t, o, _ in rows])
        with open(os.path.join(here, f"reflectance_{name}.json"), "w") as f:
            json.dump(out, f, indent=0)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/YellowThinFilms")
    main(sys.argv[1])
