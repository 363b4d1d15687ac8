"""End-to-end scenarios run identically on any engine.

Each scenario takes an engine, draws every key, ciphertext and noise vector from a
seeded numpy generator (so the inputs are identical across engines), runs one
evaluation pipeline of the reference's API and returns the raw residue rows of its
outputs.  Tests run a scenario on two engines and compare the rows bit for bit.
"""

from __future__ import annotations

import numpy as np

from vfhe_b200.arith import Polynomial, Ring
from vfhe_b200.fhe import CGGI16, CKKS_Scheme
from vfhe_b200.mlwe import CMUX, LWE, LWE_Key, MLWE, MLWE_Scheme, encrypt_lwe
from vfhe_b200.native import use_engine


def rows_of(ct: MLWE) -> np.ndarray:
    return np.stack([ct.component_rows(i) for i in range(ct.r + 1)])


def masks_of(ct: MLWE) -> list[int]:
    return [ct.component(i).rns_mask for i in range(ct.r + 1)]


def _msg(ring: Ring, rng, bound: int = 2**20) -> Polynomial:
    return Polynomial(ring).from_array([int(v) for v in rng.integers(-bound, bound, ring.N)])


def keyswitch(engine, N=256, L=4, special=1, seed=11) -> dict:
    with use_engine(engine):
        rng = np.random.default_rng(seed)
        R = Ring(N, prime_size=[50] * (L + special), split_degree=1)
        s = MLWE_Scheme(R, special_primes=special, max_lvl=L)
        k1 = s.key_gen_sparse(N // 8, 3.2, rng=rng)
        k2 = s.key_gen_sparse(N // 8, 3.2, rng=rng)
        ct = s.sample(_msg(s.ring, rng), k1, rng=rng)
        ksk = s.gen_ksk(k2, k1, rng=rng)
        out = s.keyswitch(ct, ksk)
        return {"ct": rows_of(ct), "out": rows_of(out), "mask": masks_of(out)}


def multiply(engine, N=256, L=4, special=1, seed=12) -> dict:
    with use_engine(engine):
        rng = np.random.default_rng(seed)
        R = Ring(N, prime_size=[50] * (L + special), split_degree=1)
        s = MLWE_Scheme(R, special_primes=special)
        key = s.key_gen_sparse(N // 8, 3.2, rng=rng)
        rlk = s.gen_rlk(key, key, rng=rng)
        c1 = s.sample(_msg(s.ring, rng, 8), key, rng=rng)
        c2 = s.sample(_msg(s.ring, rng, 8), key, rng=rng)
        tp = s.tensor_product(c1, c2)
        prod = s.multiply(c1, c2, rlk)
        return {"tensor": np.stack([p.rows() for p in tp]), "prod": rows_of(prod), "mask": masks_of(prod)}


def automorphism(engine, N=256, L=3, special=1, split=1, seed=13) -> dict:
    with use_engine(engine):
        rng = np.random.default_rng(seed)
        R = Ring(N, prime_size=[50] * (L + special), split_degree=split)
        s = MLWE_Scheme(R, special_primes=special)
        key = s.key_gen_sparse(N // 8, 3.2, rng=rng)
        ct = s.sample(_msg(s.ring, rng), key, rng=rng)
        gk = s.gen_ksk_automorphism(key, key, 5, rng=rng)
        out = s.automorphism(ct, 5, gk)
        return {"out": rows_of(out), "mask": masks_of(out)}


def ckks_pipeline(engine, N=256, n_mid=3, seed=14, steps=(1, 3)) -> dict:
    """mul -> relin -> rescale -> rotate on the configuration's prime shape."""
    with use_engine(engine):
        rng = np.random.default_rng(seed)
        R = Ring(N, prime_size=[50] + [40] * n_mid + [50], split_degree=1)
        s = CKKS_Scheme(R, scaling_factor=2**40, special_primes=1)
        key = s.key_gen_uniform_ternary(3.2, rng)
        s.rlk = s.gen_rlk(key, key, rng=rng)
        slots = N // 2
        z1 = np.sqrt(rng.random(slots)) * np.exp(2j * np.pi * rng.random(slots))
        z2 = np.sqrt(rng.random(slots)) * np.exp(2j * np.pi * rng.random(slots))
        c1 = s.encrypt(s.encode(list(z1)), key, rng=rng)
        c2 = s.encrypt(s.encode(list(z2)), key, rng=rng)
        prod = c1 * c2
        res = {"prod": rows_of(prod), "prod_mask": masks_of(prod), "delta": prod.delta}
        dec = np.array(s.decode(s.decrypt(prod, key), scaling_factor=prod.delta))
        res["mul_err"] = float(np.max(np.abs(dec - z1 * z2)))
        for k in steps:
            gk = s.gen_rotation_key(key, k, rng=rng)
            rot = s.rotate(prod, k, gk)
            res[f"rot{k}"] = rows_of(rot)
            dec = np.array(s.decode(s.decrypt(rot, key), scaling_factor=prod.delta))
            res[f"rot{k}_err"] = float(np.max(np.abs(dec - np.roll(z1 * z2, -k))))
        return res


def cmux(engine, N=256, seed=15) -> dict:
    with use_engine(engine):
        rng = np.random.default_rng(seed)
        Rq = Ring(N, prime_size=[50, 50, 50], split_degree=1)
        s = MLWE_Scheme(Rq, special_primes=1, module_rank=1, max_lvl=1)
        key = s.key_gen_sparse(64, 3.2, ternary=False, rng=rng)
        cg = CGGI16(s)
        bit = Polynomial(s.ring).from_array([1])
        sel = cg.mgsw_scheme.encrypt(bit, key, rng=rng)
        sel.to_NTT()
        a = s.sample(_msg(s.ring, rng), key, rng=rng)
        b = s.sample(_msg(s.ring, rng), key, rng=rng)
        out = CMUX(a, b, sel)
        ext = sel * a
        return {"cmux": rows_of(out), "ext": rows_of(ext)}


def cggi_bootstrap(engine, N=256, n_lwe=16, msg_prec=5, seed=16, count=2) -> dict:
    """Functional bootstrap as in the reference's test_cggi16.py, seeded."""
    with use_engine(engine):
        rng = np.random.default_rng(seed)
        Rq = Ring(N, prime_size=[50, 50, 50], split_degree=1)
        in_ring = Rq.quotient_ring(ell=2)
        out_scheme = MLWE_Scheme(Rq, special_primes=1, module_rank=1, max_lvl=1)
        in_key_s = [int(v) for v in rng.integers(0, 2, n_lwe)]
        in_lwe_key = LWE_Key(ring=in_ring, key=in_key_s, n=n_lwe)
        out_key = out_scheme.key_gen_sparse(64, 3.2, ternary=False, rng=rng)
        cg = CGGI16(out_scheme)
        bk = cg.generate_bootstrap_key(in_lwe_key, out_key, rng=rng)
        lut_size = 1 << (msg_prec - 1)
        lut = [int(v) for v in rng.integers(0, lut_size, lut_size)]
        tv = cg.LUT_packing(lut, lut_size, msg_prec)
        out_lwe_key = out_key.extract_lwe_key()
        key2 = LWE_Key(ring=in_ring, key=out_lwe_key.get_s(), n=out_lwe_key.n)
        outs, ok = [], []
        for _ in range(count):
            m = int(rng.integers(0, lut_size))
            scaled = round(m * in_ring.q_l / (1 << msg_prec)) % in_ring.q_l
            lwe = encrypt_lwe(in_ring, in_key_s, [scaled % q for q in in_ring.primes], 3.2, rng)
            out = LWE(ring=in_ring)
            cg.functional_bootstrap(out, tv, lwe, bk, torus_base=lut_size)
            ph = out.phase(key2, recompose=True)
            ok.append(round(ph * (1 << msg_prec) / in_ring.q_l) % (1 << msg_prec) == lut[m])
            outs.append(np.array(out.get_a()))
            outs.append(np.array(out.get_b())[None, :])
        return {"lwe": outs, "ok": ok}

