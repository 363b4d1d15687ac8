"""Evaluation-key files (vfhe_cuda_keyfile_*): save device-resident keys once, load them
back bit for bit.

The reference has no key serialisation (its keys live in process memory and are
regenerated each run); this is the engine's own format, written by native code in the
library (vfhe_b200/csrc/keyfile.cu): a versioned header with the key's kind, shape,
moduli and a payload checksum, then the raw rows.  Kinds:

* ``KSK``        relinearisation / Galois keys, u64 ``[D][2][L+1][N]`` (NTT domain)
* ``MGSW_BSK``   RNS CGGI16 bootstrapping key, u64 ``[n][2 L0][2][L0+1][N]`` (NTT domain)
* ``TORUS_BSK``  torus bootstrapping-key rows, u32 ``[n][2 levels][2][N]``
* ``TORUS_KSK``  torus key-switching key, u32 ``[N][levels][n+1]``
"""

from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np
import torch

from .native import Engine, EngineError, cuda_engine

KSK, MGSW_BSK, TORUS_BSK, TORUS_KSK = 1, 2, 3, 4


@dataclass
class KeyHeader:
    kind: int
    shape: tuple
    elem_bytes: int
    moduli: list = field(default_factory=list)
    aux: list = field(default_factory=lambda: [0, 0, 0, 0])


def _engine(engine: Engine | None) -> Engine:
    if engine is not None:
        return engine
    # the file functions need no GPU: load the library without the device check
    from .native import CUDA_LIB

    return Engine(CUDA_LIB, "cuda")


def _c_header(eng: Engine, h: KeyHeader):
    c = eng.ffi.new("VfheKeyHeader*")
    c.kind = h.kind
    c.elem_bytes = h.elem_bytes
    c.ndims = len(h.shape)
    for d, v in enumerate(h.shape):
        c.dims[d] = int(v)
    c.nmoduli = len(h.moduli)
    for k, q in enumerate(h.moduli):
        c.moduli[k] = int(q)
    for k, a in enumerate(h.aux):
        c.aux[k] = int(a)
    return c


def _py_header(c) -> KeyHeader:
    return KeyHeader(kind=int(c.kind), shape=tuple(int(c.dims[d]) for d in range(c.ndims)),
                     elem_bytes=int(c.elem_bytes), moduli=[int(c.moduli[k]) for k in range(c.nmoduli)],
                     aux=[int(c.aux[k]) for k in range(4)])


def write_host(path: str | os.PathLike, header: KeyHeader, data: np.ndarray, engine: Engine | None = None) -> None:
    """Write a host array (uint64 or uint32, C order, shape == header.shape)."""
    eng = _engine(engine)
    arr = np.ascontiguousarray(data)
    if tuple(arr.shape) != tuple(header.shape) or arr.itemsize != header.elem_bytes:
        raise ValueError("array shape or element size does not match the header")
    if eng.lib.vfhe_cuda_keyfile_write(os.fsencode(path), _c_header(eng, header), eng.ffi.from_buffer(arr)) != 0:
        eng.check("keyfile_write")
        raise EngineError("keyfile_write")


def read_header(path: str | os.PathLike, engine: Engine | None = None) -> KeyHeader:
    eng = _engine(engine)
    c = eng.ffi.new("VfheKeyHeader*")
    if eng.lib.vfhe_cuda_keyfile_read_header(os.fsencode(path), c) != 0:
        eng.check("keyfile_read_header")
        raise EngineError("keyfile_read_header")
    return _py_header(c)


def read_host(path: str | os.PathLike, engine: Engine | None = None) -> tuple[KeyHeader, np.ndarray]:
    """Header and payload (uint64 or uint32 array of the stored shape), checksum verified."""
    eng = _engine(engine)
    h = read_header(path, eng)
    dtype = np.uint64 if h.elem_bytes == 8 else np.uint32
    arr = np.empty(h.shape, dtype=dtype)
    c = eng.ffi.new("VfheKeyHeader*")
    if eng.lib.vfhe_cuda_keyfile_read(os.fsencode(path), c, eng.ffi.from_buffer(arr), arr.nbytes) != 0:
        eng.check("keyfile_read")
        raise EngineError("keyfile_read")
    return _py_header(c), arr


def save(path: str | os.PathLike, key: torch.Tensor, kind: int, moduli=(), aux=(0, 0, 0, 0),
         engine: Engine | None = None) -> None:
    """Write a device key tensor (int64 rows of u64 residues, or int32 torus values)."""
    host = key.detach().cpu().numpy()
    host = host.view(np.uint64) if host.itemsize == 8 else host.view(np.uint32)
    aux = list(aux) + [0] * (4 - len(aux))
    write_host(path, KeyHeader(kind, tuple(host.shape), host.itemsize, list(moduli), aux), host, engine)


def load(path: str | os.PathLike, device: str = "cuda", engine: Engine | None = None) -> tuple[KeyHeader, torch.Tensor]:
    """Read a key file back to a device tensor of the stored shape (int64 / int32 view)."""
    h, arr = read_host(path, engine or cuda_engine())
    t = torch.from_numpy(arr.view(np.int64) if arr.itemsize == 8 else arr.view(np.int32))
    return h, t.to(device)
