"""Generate the golden fixtures of the plain FP64 step from the reference itself.

Each case is a seeded synthetic deck (frehdc_b200.deck) run by the reference
program built from its own sources, twice:
  <case>_ssor.npz    oracle/_ref/frehd_ref: the reference as shipped, laspack's
                     CGIter with SSORPrecond from x = 0 (nsfunctions.c:1004-1017)
  <case>_jacobi.npz  oracle/_ref/frehd_ref_jacobi: the same program with
                     laspack's JacobiPrecond handed to that CGIter call, the
                     preconditioner of the device solve
A fixture keeps, for the final state of the run:
  * the deck's fingerprint (SHA-256 of its fine bottoms, initial surface,
    initial scalar and tide series), so a change of the generator is caught;
  * every field at 2048 seeded cell positions (exact doubles);
  * per-field checksums over all interior cells: sum, sum of squares, min, max.

Cases:
  c1_128      128 x 128, dx 10 m, dt 1 s, 200 steps, n 0.03 (the CPU case)
  c2crop_512  the 512 x 512 window of the 4096 x 4096 deck (dx 2 m, dt 0.5 s,
              ~30 % dry, n 0.025) along its tidal edge, 1000 steps (the step
              count of the 4096 x 4096 workload), with the scalar plume
              centred in the window

Run from the repository root where the reference sources are present (the two
reference runs of a case run side by side; the 512 x 512 case takes minutes):
    python tests/golden/make_golden.py [case ...]
"""
from __future__ import annotations

import hashlib
import math
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

from frehdc_b200 import deck as D  # noqa: E402

FIELDS = ["surf", "uuXP", "vvYP", "S", "depth", "cellV"]
N_SAMPLES = 2048
SAMPLE_SEED = 20240611


def c1_spec() -> D.DeckSpec:
    return D.DeckSpec(nx=128, ny=128, dx=10.0, dt=1.0, steps=200, manning_n=0.03, seed=1234)


def c2crop_spec() -> D.DeckSpec:
    full = D.DeckSpec(nx=4096, ny=4096, dx=2.0, dt=0.5, steps=1000, seed=2024, dry_frac=0.3,
                      manning_n=0.025)
    return full.replace(nx=512, ny=512, crop=(0, 4096 - 512, 4096, 4096), scalar_in_window=True)


CASES = {"c1_128": c1_spec, "c2crop_512": c2crop_spec}
PRECONDS = ("jacobi", "ssor")


def fingerprint(deck) -> str:
    h = hashlib.sha256()
    for a in (deck.zf, deck.surf0, deck.S0, D.tide_series(deck)):
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    return h.hexdigest()


def sample_index(n_cells: int) -> np.ndarray:
    rng = np.random.default_rng(SAMPLE_SEED)
    return np.sort(rng.choice(n_cells, size=min(N_SAMPLES, n_cells), replace=False))


def checksums(a: np.ndarray) -> np.ndarray:
    a = np.asarray(a, dtype=np.float64)
    return np.array([math.fsum(a), math.fsum(a * a), a.min(), a.max()])


def fixture_path(case: str, precond: str) -> str:
    return os.path.join(HERE, f"{case}_{precond}.npz")


def load(case: str, precond: str) -> dict:
    with np.load(fixture_path(case, precond)) as z:
        return {k: z[k] for k in z.files}


def main(cases: list[str]) -> int:
    from concurrent.futures import ThreadPoolExecutor

    from oracle import refrun
    if not refrun.build():
        print("the reference oracle binaries are not available", file=sys.stderr)
        return 1
    for case in cases or list(CASES):
        spec = CASES[case]()
        deck = D.make_deck(spec)
        N = spec.nx * spec.ny
        idx = sample_index(N)
        with tempfile.TemporaryDirectory() as tmp:
            path = os.path.join(tmp, case)
            D.write_reference_deck(deck, path)

            def one(precond):
                return refrun.run(path, spec.steps, os.path.join(tmp, f"final_{precond}.bin"),
                                  precond=precond)
            with ThreadPoolExecutor(len(PRECONDS)) as ex:
                states = dict(zip(PRECONDS, ex.map(one, PRECONDS)))
        for precond in PRECONDS:
            st = states[precond]
            out = {"fingerprint": np.array(fingerprint(deck)), "steps": np.array(spec.steps),
                   "idx": idx, "precond": np.array(precond)}
            for f in FIELDS:
                a = st[f][:N]
                out[f] = a[idx]
                out[f + "_sums"] = checksums(a)
            np.savez_compressed(fixture_path(case, precond), **out)
            print(case, precond, "steps", spec.steps, "volume", out["cellV_sums"][0])
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
