"""Known-answer vectors from the reference's own code (tests/golden/ref_kat.npz).

Runs oracle/_ref/libref_kat.so -- the reference's unmodified headers
(random.h, luminance.h, Reservoir.h, Camera.h, sample_emitter.h and the
cut ranges of path_gen.h, Emitter.h and brdf.cu) compiled by
`make -C oracle ref` where the CrisOptix sources are present -- on seeded
inputs that include the edge values the functions special-case (zero
luminance, NaN and infinite weights and jacobians, coincident points,
window clamping at unsigned wrap-around), and stores inputs and answers.

    make -C oracle ref && python tests/golden/make_ref_kat.py
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import kat_cases  # noqa: E402

OUT = os.path.join(HERE, "ref_kat.npz")


def main():
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_kat.so"))
    lib.ref_kat.restype = ctypes.c_int
    lib.ref_kat.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p]
    lib.ref_kat_emitter.restype = ctypes.c_int
    lib.ref_kat_emitter.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p]
    data = {}
    for name, fn in kat_cases.FUNCTIONS.items():
        inp = kat_cases.inputs(fn, seed=fn)
        data[f"{name}_in"] = inp
        data[f"{name}_out"] = kat_cases.run(lambda f, i, n, o: lib.ref_kat(f, i, n, o), fn, inp)
    ems, faces, states = kat_cases.emitter_case(seed=77)
    out, st = kat_cases.run_emitter(lib.ref_kat_emitter, ems, faces, states)
    data.update(emitter_table=ems, emitter_faces=faces, emitter_states=states, emitter_out=out,
                emitter_state_out=st)
    np.savez_compressed(OUT, **data)
    print(f"wrote {OUT}: " + ", ".join(f"{k} {v.shape}" for k, v in data.items()))


if __name__ == "__main__":
    main()
