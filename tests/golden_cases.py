"""Loader for tests/golden/reference_cases.npz (made by tests/golden/make_golden.py)."""
from __future__ import annotations

import os

import numpy as np

from qlassical_b200._lib import GATE_INSTR_DTYPE, MATRIX_ENTRY_DTYPE
from qlassical_b200.ir import IRModule, UnitaryPool

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_cases.npz")


class Case:
    def __init__(self, name, z):
        self.name = name
        self.n = int(z[f"{name}/n"])
        prog = np.frombuffer(z[f"{name}/prog"].tobytes(), dtype=GATE_INSTR_DTYPE)
        meta = np.frombuffer(z[f"{name}/pool_meta"].tobytes(), dtype=MATRIX_ENTRY_DTYPE)
        self.module = IRModule(self.n, unitary_pool=UnitaryPool.from_arrays(z[f"{name}/pool_data"], meta))
        self.module.set_program(prog)
        init = z[f"{name}/init"]
        self.init = init if init.size else None
        self.seed = int(z[f"{name}/seed"])
        self.expected = z[f"{name}/expected"]
        self.meas = [int(x) for x in z[f"{name}/meas"]]


def load_cases():
    z = np.load(PATH)
    names = sorted({k.split("/")[0] for k in z.files})
    return [Case(nm, z) for nm in names]
