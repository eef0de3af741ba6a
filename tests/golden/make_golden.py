"""Generate tests/golden/rng_golden.json.

Run in the build container, where the reference tree is mounted:
    python tests/golden/make_golden.py /root/reference/src3_mpi_cfitsio

It reads the L'Ecuyer-Cote constants straight from the reference's
ecuyer_cote_mod.f90 (lines 14-17: a1, a1vw, a1w, a2, a2vw, a2w, m1, m2) and
evaluates, with Python's exact big integers and independently of the C
oracle, the recurrences the reference implements:
  * random_large_integer (ecuyer_cote_mod.f90:252-293) as s <- a*s mod m,
    z = s1 - s2 (+ m1 - 1 if z < 1), xi = z * 4.656613057e-10
    (random_standard_uniform_mod.f90:339);
  * set_all_seeds (:350-395): generator g starts at a^((g-1)*2^50) * seed;
  * reinitialize_current_generator(1) (:335-337): next block = a^(2^30) * block.
The fixture stores the constants, whether a1w = a1^(2^30), a1vw = a1^(2^50)
hold (they must), and the first draws of several packets' streams for the
seeds the reference uses (user_set_all(12345678,87654321,g), newtts.f90:105).
The GPU box never reads the reference: tests load only this JSON.
"""
from __future__ import annotations

import json
import os
import re
import sys


def parse_constants(src_dir: str) -> dict:
    text = open(os.path.join(src_dir, "ecuyer_cote_mod.f90")).read()
    consts = {}
    for name in ("a1", "a1vw", "a1w", "a2", "a2vw", "a2w", "m1", "m2", "n_generators"):
        m = re.search(r"\b%s\s*=\s*(\d+)" % name, text)
        consts[name] = int(m.group(1))
    return consts


def stream_seeds(c, seed1, seed2, generator, block):
    g1, g2 = seed1, seed2
    for _ in range(2, generator + 1):
        g1 = c["a1vw"] * g1 % c["m1"]
        g2 = c["a2vw"] * g2 % c["m2"]
    s1 = pow(c["a1w"], block, c["m1"]) * g1 % c["m1"]
    s2 = pow(c["a2w"], block, c["m2"]) * g2 % c["m2"]
    return s1, s2


def draws(c, s1, s2, n):
    out = []
    for _ in range(n):
        s1 = c["a1"] * s1 % c["m1"]
        s2 = c["a2"] * s2 % c["m2"]
        z = s1 - s2
        if z < 1:
            z += c["m1"] - 1
        out.append((z, float(z) * 4.656613057e-10))
    return out


def main(src_dir: str):
    c = parse_constants(src_dir)
    checks = {
        "a1w_is_a1_pow_2_30": pow(c["a1"], 2 ** 30, c["m1"]) == c["a1w"],
        "a2w_is_a2_pow_2_30": pow(c["a2"], 2 ** 30, c["m2"]) == c["a2w"],
        "a1vw_is_a1_pow_2_50": pow(c["a1"], 2 ** 50, c["m1"]) == c["a1vw"],
        "a2vw_is_a2_pow_2_50": pow(c["a2"], 2 ** 50, c["m2"]) == c["a2vw"],
    }
    cases = []
    for (g, block) in [(1, 0), (1, 1), (1, 2), (1, 999), (2, 0), (5, 12345), (32, 10 ** 8 - 1),
                       (1, 10 ** 9 + 7)]:
        s1, s2 = stream_seeds(c, 12345678, 87654321, g, block)
        d = draws(c, s1, s2, 8)
        cases.append({"seed1": 12345678, "seed2": 87654321, "generator": g, "block": block,
                      "s1": s1, "s2": s2, "z": [z for z, _ in d], "xi": [x for _, x in d]})
    out = {"source": "src3_mpi_cfitsio/ecuyer_cote_mod.f90:14-17", "constants": c, "checks": checks,
           "cases": cases}
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "rng_golden.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(path, checks)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <path of the reference's src3_mpi_cfitsio directory>")
    main(sys.argv[1])
