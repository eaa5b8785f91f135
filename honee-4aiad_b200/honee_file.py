"""HONEE's binary solution files (src/honee-file.c:136-232): checkpoints written by HoneeWriteBinaryVec and read by
HoneeLoadBinaryVec, the format of the reference's tests/output/*.bin.

Layout, big-endian like PETSc's binary viewer:
  HONEE file   int32 token (0x0CEEDF32 for 32-bit PetscInt, 0x0CEEDF64 for 64-bit, 0x0CEEDF00 for the older form read as
               32-bit), step number (int32 or int64), time (float64), then a PETSc Vec: class id and length (int32 each, or
               int64 each with 64-bit indices), then the values (float64)
  legacy Vec   the PETSc Vec alone (class id 1211214, length, values), step 0 and time 0

The values are a global vector in the writer's node ordering: HONEE's are DMPlex's, this package's the box mesh's
(node-interleaved, essential DOFs removed), so a file moves between the two only through a permutation; within one
ordering it is a checkpoint (hb_ts_get_state / hb_ts_set_state, or the explicit stepper's).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

TOKEN_32 = 0x0CEEDF32
TOKEN_64 = 0x0CEEDF64
TOKEN = 0x0CEEDF00
VEC_FILE_CLASSID = 1211214


@dataclass
class HoneeFile:
    values: np.ndarray
    step: int
    time: float
    int64: bool


def read(path: str) -> HoneeFile:
    raw = open(path, "rb").read()
    token = int(np.frombuffer(raw[:4], dtype=">i4")[0])
    if token in (TOKEN_32, TOKEN_64, TOKEN):
        wide = token == TOKEN_64
        itype, isz = (">i8", 8) if wide else (">i4", 4)
        pos = 4
        step = int(np.frombuffer(raw[pos:pos + isz], dtype=itype)[0])
        pos += isz
        time = float(np.frombuffer(raw[pos:pos + 8], dtype=">f8")[0])
        pos += 8
        classid, length = (int(v) for v in np.frombuffer(raw[pos:pos + 2 * isz], dtype=itype))
        pos += 2 * isz
    else:  # the Vec alone; 64-bit indices split the class id over two int32 words (VecLoad_Binary)
        step, time = 0, 0.0
        if token == VEC_FILE_CLASSID:
            wide, classid = False, token
            length = int(np.frombuffer(raw[4:8], dtype=">i4")[0])
            pos = 8
        else:
            wide = True
            classid, length = (int(v) for v in np.frombuffer(raw[:16], dtype=">i8"))
            pos = 16
    if classid != VEC_FILE_CLASSID:
        raise ValueError(f"{path}: not a HONEE solution file or PETSc Vec (class id {classid})")
    if len(raw) != pos + 8 * length:
        raise ValueError(f"{path}: {len(raw) - pos} value bytes for a Vec of length {length}")
    return HoneeFile(np.frombuffer(raw[pos:], dtype=">f8").astype(np.float64), step, time, wide)


def write(path: str, values, step: int = 0, time: float = 0.0, int64: bool = False) -> None:
    """HoneeWriteBinaryVec: token, step, time, then the Vec (class id, length, big-endian values)."""
    v = np.ascontiguousarray(values, dtype=np.float64)
    itype = ">i8" if int64 else ">i4"
    with open(path, "wb") as f:
        f.write(np.array([TOKEN_64 if int64 else TOKEN_32], dtype=">i4").tobytes())
        f.write(np.array([step], dtype=itype).tobytes())
        f.write(np.array([time], dtype=">f8").tobytes())
        f.write(np.array([VEC_FILE_CLASSID, v.size], dtype=itype).tobytes())
        f.write(v.astype(">f8").tobytes())


def free_values(state: np.ndarray, essential: np.ndarray | None) -> np.ndarray:
    """The global vector of a full L-vector state: the entries that are not essential DOFs, in L-vector order."""
    if essential is None or len(essential) == 0:
        return np.asarray(state)
    keep = np.ones(np.asarray(state).size, dtype=bool)
    keep[np.asarray(essential)] = False
    return np.asarray(state)[keep]


def expand(values: np.ndarray, l_size: int, essential: np.ndarray | None, essential_values=None) -> np.ndarray:
    """Inverse of free_values: scatter a global vector into an L-vector with the essential values inserted."""
    q = np.zeros(l_size)
    keep = np.ones(l_size, dtype=bool)
    if essential is not None and len(essential):
        keep[np.asarray(essential)] = False
        q[np.asarray(essential)] = 0.0 if essential_values is None else essential_values
    q[keep] = values
    return q
