"""Child-process driver of the reference's own CKKS and CGGI16 classes -- TEST INFRASTRUCTURE.

Run with the reference's Python packages on the path (oracle/build_dropin.py) and
`VFHE_ENGINE` naming the engine; nothing here is the engine's own Python mirror:

    python tests/dropin_driver.py <scenario> make   <dir>   # reference engine
    python tests/dropin_driver.py <scenario> inject <dir>   # engine under test

`make` builds keys and ciphertexts with the reference's classes on the running engine,
dumps every input residue row to <dir>/inputs.npz, runs the operation and dumps the
outputs to <dir>/out_<engine>.npz.  `inject` builds the same objects through the same
calls (their random draws differ per engine, as the reference's two engines differ),
overwrites every input row with the dumped ones, runs the same operation and dumps its
outputs.  Equal outputs then mean the reference's orchestration gives the same residues
on both engines.

Scenarios (seeded with numpy PCG64):
  ckks  the CKKS configuration: N = 2^14, primes [50] + [40]*8 + [50] (one special),
        scale 2^40, ternary secret; two ciphertexts of unit-disk slots;
        `c1 * c2` (CKKS_Ciphertext.__mul__: multiply, relinearise, rescale;
        modules/fhe/python/src/vfhe/fhe/ckks.py:227-241) then `rotate` by 2^5
        (ckks.py:110-119).
  cggi  CGGI16.functional_bootstrap (modules/fhe/python/src/vfhe/fhe/cggi16.py:115-128)
        at N = 1024, [50, 50, 50] with one special prime, a binary LWE key of
        dimension 630, 5-bit LUT precision, on two LWEs.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

SEED = 20260


def _rows(handle, ffi) -> list[np.ndarray]:
    p = ffi.cast("RNS_Polynomial", handle)
    N = int(p.ntt.N)
    out = []
    for i in range(int(p.allocated_l)):
        if (int(p.rns_mask) >> i) & 1:
            out.append(np.frombuffer(ffi.buffer(p.coeffs[i], 8 * N), dtype=np.uint64).copy())
    return out


def _set_rows(handle, rows: list[np.ndarray], ffi) -> list[np.ndarray]:
    p = ffi.cast("RNS_Polynomial", handle)
    N = int(p.ntt.N)
    k = 0
    for i in range(int(p.allocated_l)):
        if (int(p.rns_mask) >> i) & 1:
            ffi.memmove(p.coeffs[i], np.ascontiguousarray(rows[k], dtype=np.uint64).tobytes(), 8 * N)
            k += 1
    assert k == len(rows)
    return rows[k:]


def _mlwe_polys(handle, ffi) -> list:
    m = ffi.cast("RNS_MLWE", handle)
    return [m.a[j] for j in range(int(m.r))] + [m.b]


def _set_polys(mlwe_set, ffi) -> list:
    """Every polynomial handle of an MLWE_Set's C copies (the arrays the C key switch reads)."""
    out = []
    for j, comp in enumerate(mlwe_set.mlwe):
        if comp is None:
            continue
        arr = ffi.cast("RNS_MLWE *", mlwe_set.obj[j])
        for d in range(len(comp)):
            out += _mlwe_polys(arr[d], ffi)
    return out


def _dump(polys: list, ffi) -> np.ndarray:
    return np.concatenate([np.stack(_rows(h, ffi)) for h in polys])


def _load(polys: list, stacked: np.ndarray, ffi) -> None:
    k = 0
    for h in polys:
        n = len(_rows(h, ffi))
        _set_rows(h, list(stacked[k:k + n]), ffi)
        k += n
    assert k == stacked.shape[0]


def _lwe_rows(obj, ffi, n: int, l: int) -> np.ndarray:
    w = ffi.cast("LWE", obj)
    a = np.stack([np.frombuffer(ffi.buffer(w.a[j], 8 * n), dtype=np.uint64).copy() for j in range(l)])
    b = np.frombuffer(ffi.buffer(w.b, 8 * l), dtype=np.uint64).copy()
    return np.concatenate([a.reshape(-1), b])


def _set_lwe_rows(obj, ffi, n: int, l: int, flat: np.ndarray) -> None:
    w = ffi.cast("LWE", obj)
    for j in range(l):
        ffi.memmove(w.a[j], np.ascontiguousarray(flat[j * n:(j + 1) * n]).tobytes(), 8 * n)
    ffi.memmove(w.b, np.ascontiguousarray(flat[l * n:]).tobytes(), 8 * l)


def ckks(mode: str, d: Path) -> dict:
    from vfhe.arith import Ring
    from vfhe.fhe import CKKS_Scheme
    from vfhe.misc.libvfhe import ffi
    from vfhe.mlwe.mlwe import MLWE_Key

    rng = np.random.default_rng(SEED)
    N, step = 2**14, 32
    R = Ring(N, prime_size=[50] + [40] * 8 + [50], split_degree=1)
    s = CKKS_Scheme(R, scaling_factor=2**40, special_primes=1)
    key = MLWE_Key([[int(v) for v in rng.integers(-1, 2, N)]], 3.2, s)
    rlk = s.gen_rlk(key, key, lvl=0)
    s.rlk = [rlk]
    gk = s.gen_ksk_automorphism(key, key, pow(5, step, 2 * N), lvl=1)
    z = [np.sqrt(rng.random(N // 2)) * np.exp(2j * np.pi * rng.random(N // 2)) for _ in range(2)]
    c1, c2 = (s.encrypt(s.encode([complex(v) for v in zz]), key) for zz in z)
    groups = {"rlk": _set_polys(rlk, ffi), "gk": _set_polys(gk, ffi),
              "c1": _mlwe_polys(c1.obj, ffi), "c2": _mlwe_polys(c2.obj, ffi)}
    if mode == "make":
        np.savez(d / "inputs.npz", **{k: _dump(v, ffi) for k, v in groups.items()})
    else:
        inp = np.load(d / "inputs.npz")
        for k, v in groups.items():
            _load(v, inp[k], ffi)
    prod = c1 * c2
    rot = s.rotate(prod, step, gk)
    out = {"prod": _dump(_mlwe_polys(prod.obj, ffi), ffi), "rot": _dump(_mlwe_polys(rot.obj, ffi), ffi)}
    info = {}
    if mode == "make":
        want = np.roll(z[0] * z[1], -step)
        got = np.array(s.decode(s.decrypt(rot, key), scaling_factor=rot.delta))
        info["decoded_max_error"] = float(np.abs(got - want).max())
    return out, info


def cggi(mode: str, d: Path) -> dict:
    from vfhe.arith import Ring
    from vfhe.fhe import CGGI16
    from vfhe.misc.libvfhe import ffi
    from vfhe.mlwe.lwe import LWE, LWE_Key
    from vfhe.mlwe.mlwe import MLWE_Key, MLWE_Scheme

    rng = np.random.default_rng(SEED + 1)
    n, N, t, count = 630, 1024, 16, 2
    Rq = Ring(N, prime_size=[50, 50, 50], split_degree=1)
    in_ring = Rq.quotient_ring(ell=2)
    s = MLWE_Scheme(Rq, special_primes=1, module_rank=1, max_lvl=1)
    key_s = [int(v) for v in rng.integers(0, 2, n)]
    in_key = LWE_Key(ring=in_ring, key=key_s, n=n)
    ffi.cast("LWE_Key", in_key.obj).sigma = 3.2  # lwe_alloc_key leaves sigma unset (lwe.c:6-18)
    out_list = [0] * N
    for i in rng.choice(N, 64, replace=False):
        out_list[int(i)] = 1
    out_key = MLWE_Key([out_list], 3.2, s)
    cg = CGGI16(s)
    bk = cg.generate_bootstrap_key(in_key, out_key)
    lut = [int(v) for v in rng.integers(0, t, t)]
    tv = cg.LUT_packing(lut, t, 5)
    msgs = [int(v) for v in rng.integers(0, t, count)]
    lwes = [LWE(ring=in_ring, m=[round(m * in_ring.q_l / 32) % q for q in in_ring.primes], key=in_key)
            for m in msgs]
    bk_polys = [h for mg in bk.bk for c in mg.obj for h in _mlwe_polys(c.obj, ffi)]
    if mode == "make":
        np.savez(d / "inputs.npz", bk=_dump(bk_polys, ffi),
                 lwe=np.stack([_lwe_rows(x.obj, ffi, n, 2) for x in lwes]))
    else:
        inp = np.load(d / "inputs.npz")
        _load(bk_polys, inp["bk"], ffi)
        for x, flat in zip(lwes, inp["lwe"]):
            _set_lwe_rows(x.obj, ffi, n, 2, flat)
    outs, info = [], {}
    okey = out_key.extract_lwe_key()
    key2 = LWE_Key(ring=in_ring, key=okey.get_s(), n=okey.n)
    dec = []
    for x in lwes:
        o = LWE(ring=in_ring)
        cg.functional_bootstrap(o, tv, x, bk, torus_base=t)
        outs.append(_lwe_rows(o.obj, ffi, N, 2))
        ph = o.phase(key2, recompose=True)
        dec.append(int(round(ph * 32 / in_ring.q_l) % 32))
    info["decrypted"] = dec
    info["expected"] = [lut[m] for m in msgs]
    return {"lwe_out": np.stack(outs)}, info


def main() -> None:
    scenario, mode, d = sys.argv[1], sys.argv[2], Path(sys.argv[3])
    from vfhe.misc.libvfhe import active_engine

    out, info = {"ckks": ckks, "cggi": cggi}[scenario](mode, d)
    eng = active_engine()
    np.savez(d / f"out_{eng}.npz", **out)
    import json

    (d / f"info_{eng}.json").write_text(json.dumps(info))
    print(f"{scenario} {mode} on {eng}: ok")


if __name__ == "__main__":
    main()
