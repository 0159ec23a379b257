"""Writes the expected object model of every HiG fixture in this folder, as the reference's own
reader builds it: <name>.ref.json, produced by oracle/_ref/libhigref.so (ref_hig_json, the
reference's HiGInput::construct_input_config compiled from its sources by `make -C oracle ref`).
Also checks that the reference rejects every file under bad/, and writes
fit_update.updated.ref.json: the model after HiGInput::update_params sets the fixture's fit
parameters (key order) to FIT_VALUES.

    python tests/golden/hig/gen_hig_golden.py

Needs the reference tree (the oracle/_ref build); the committed .ref.json files let the tests
run without it.
"""
from __future__ import annotations

import ctypes
import glob
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(os.path.dirname(HERE)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libhigref.so")


def ref_reader():
    lib = ctypes.CDLL(REF_LIB)
    lib.ref_hig_json.restype = ctypes.c_long
    lib.ref_hig_json.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_long]
    buf = ctypes.create_string_buffer(1 << 22)

    def read(path):
        # the reference opens included files relative to the working directory
        cwd = os.getcwd()
        os.chdir(os.path.dirname(os.path.abspath(path)))
        try:
            n = lib.ref_hig_json(os.fsencode(os.path.abspath(path)), buf, len(buf))
        finally:
            os.chdir(cwd)
        if n == -2:
            raise RuntimeError("JSON buffer too small")
        return json.loads(buf.value.decode()) if n >= 0 else None

    return read


def fit_values(n):
    """The values the update test gives the i-th fit parameter (key order)."""
    return [1.5 + 0.25 * i for i in range(n)]


def ref_updated(path, keys, vals):
    lib = ctypes.CDLL(REF_LIB)
    lib.ref_hig_json_updated.restype = ctypes.c_long
    lib.ref_hig_json_updated.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_char_p),
                                         ctypes.POINTER(ctypes.c_double), ctypes.c_int,
                                         ctypes.c_char_p, ctypes.c_long]
    buf = ctypes.create_string_buffer(1 << 22)
    ck = (ctypes.c_char_p * len(keys))(*[k.encode() for k in keys])
    cv = (ctypes.c_double * len(vals))(*vals)
    n = lib.ref_hig_json_updated(os.fsencode(path), ck, cv, len(keys), buf, len(buf))
    if n < 0:
        raise RuntimeError(f"the reference refused the update of {path} ({n})")
    return json.loads(buf.value.decode())


def main():
    read = ref_reader()
    for path in sorted(glob.glob(os.path.join(HERE, "*.hig"))):
        d = read(path)
        if d is None:
            sys.exit(f"the reference rejected {path}")
        out = path[:-4] + ".ref.json"
        with open(out, "w") as f:
            json.dump(d, f, indent=1, sort_keys=True)
            f.write("\n")
        print("wrote", os.path.relpath(out, ROOT))
    path = os.path.join(HERE, "fit_update.hig")
    keys = sorted(read(path)["fitparams"])
    d = ref_updated(path, keys, fit_values(len(keys)))
    with open(path[:-4] + ".updated.ref.json", "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)
        f.write("\n")
    print("wrote", os.path.relpath(path[:-4] + ".updated.ref.json", ROOT))
    for path in sorted(glob.glob(os.path.join(HERE, "bad", "*.hig"))):
        if read(path) is not None:
            sys.exit(f"the reference accepted {path}, expected a rejection")
    print("the reference rejects all", len(glob.glob(os.path.join(HERE, "bad", "*.hig"))), "files under bad/")


if __name__ == "__main__":
    main()
