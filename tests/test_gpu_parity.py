"""GPU parity of the hot path against the oracle (CPU restatement of the reference).

Superblocks are captured from oracle sweeps (warm-up, left_to_right and
right_to_left steps, with and without t2/J2) and fed through the C-ABI.
Tolerances (complex FP64 throughout): H.psi element-wise max|dx|/max|x| <= 1e-13;
Lanczos energy |dE/E| <= 1e-12; truncation spectrum <= 1e-12 absolute with the
kept count identical; renormalised operators and wave transforms <= 1e-12
relative to their largest element.
"""
import numpy as np
import pytest

import orc
from _capture import parse_oracle_capture
from tsc_tri_t1t2j1j2_b200 import Context

CASES = [
    # (Nx, t2, J2, kept, capture index): warm-up, LR sweep, RL sweep steps
    (4, 0.0, 0.0, 60, 3),
    (4, 0.3, 0.036, 60, 6),
    (4, 0.3, 0.036, 60, 14),
    (4, 0.0, 0.0, 80, 22),
]


def oracle_capture(Nx, t2, J2, kept, step):
    cfg = orc.RunConfig(Nx=Nx, Ny=4, t1=1.0, t2=t2, J1=0.4, J2=J2, kept_min=kept, kept_warm=kept,
                        sweeps=[kept], lanzero=1e-10)
    o = orc.Oracle(cfg, capture_step=step)
    o.run()
    return cfg, parse_oracle_capture(*o.capture())


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module", params=CASES, ids=lambda c: f"Nx{c[0]}_t2{c[1]}_m{c[3]}_s{c[4]}")
def captured(request):
    Nx, t2, J2, kept, step = request.param
    cfg, cap = oracle_capture(Nx, t2, J2, kept, step)
    ctx = Context(Nx, 4, 1.0, t2, 0.4, J2)
    ctx.set_superblock(cap["sys"], cap["env"], cap["sys_bs"], cap["env_bs"], cap["psi0"])
    yield cfg, cap, ctx
    ctx.close()


@pytest.mark.gpu
def test_hpsi_matches_oracle(captured):
    _, cap, ctx = captured
    out = ctx.model_wave(cap["psi0"].vec)
    assert rel(out, cap["hpsi"].vec) <= 1e-13


@pytest.mark.gpu
def test_lanczos_matches_oracle(captured):
    _, cap, ctx = captured
    vec, e0, iters = ctx.lanczos_memo_new(cap["psi0"].vec, 1e-10)
    assert abs(e0 - cap["e0"]) <= 1e-12 * abs(cap["e0"])
    assert abs(iters - cap["iters"]) <= 1
    ov = abs(np.vdot(vec, cap["gs"].vec))
    assert abs(ov - 1.0) <= 1e-9


@pytest.mark.gpu
def test_truncation_matches_oracle(captured):
    cfg, cap, ctx = captured
    side = 0 if cap["sys_side"] else 1
    if cap["trun"].num == 0 or len(cap["spectrum"]) == 0:
        pytest.skip("warm-up step kept every state (identity truncation)")
    r = ctx.get_truncation_operator(side, cap["gs"].vec, cfg.kept_min, cfg.sweeps[0], 1.0000000036274937e-15)
    n = len(cap["spectrum"])
    assert np.max(np.abs(r["spectrum"][:n] - cap["spectrum"])) <= 1e-12
    assert r["num_state"] == cap["num_state"]
    assert abs(r["err"] - cap["err"]) <= 1e-12
    assert abs(r["entropy"] - cap["ent"]) <= 1e-10
    # U is fixed up to a phase per column, and kept states beyond the rank of rho
    # (zero weight, ordered by rounding noise in any eigensolver) are arbitrary:
    # compare the projectors onto the kept states of non-negligible weight.
    t = r["trun"]
    den = {(int(s[0]), int(s[1])): m for s, m in zip(cap["den"].subs, cap["den"].mats)}

    def significant(block):
        out = {}
        for sub, u in zip(block.subs, block.mats):
            rho = den[(int(sub[0]), int(sub[1]))]
            w = np.real(np.einsum("ia,ij,ja->a", u.conj(), rho, u))
            keep = u[:, w > 1e-10]
            out[(int(sub[0]), int(sub[1]))] = keep @ keep.conj().T
        return out

    pa, pb = significant(t), significant(cap["trun"])
    for key in set(pa) | set(pb):
        a = pa.get(key)
        b = pb.get(key)
        if a is None or b is None:
            z = a if a is not None else b
            assert np.max(np.abs(z), initial=0.0) <= 1e-9
            continue
        assert np.max(np.abs(a - b)) <= 1e-9


@pytest.mark.gpu
def test_density_matrix_entry_and_levels(captured):
    """tsc_density_matrix (Get_density_matrix_*_new) against the oracle's density
    matrix (<= 1e-13 of its largest element), tsc_truncation_operator on that
    matrix bit-identical to tsc_truncate, and levels = 2 equal to the average of
    the two waves' unnormalised density matrices computed in numpy."""
    cfg, cap, ctx = captured
    side = 0 if cap["sys_side"] else 1
    gs = cap["gs"]
    den = ctx.get_density_matrix(side, gs.vec)
    ref = {(int(s[0]), int(s[1])): m for s, m in zip(cap["den"].subs, cap["den"].mats)}
    scale = max(np.max(np.abs(m)) for m in ref.values())
    assert den.num == len(ref)
    for sub, m in zip(den.subs, den.mats):
        assert np.max(np.abs(m - ref[(int(sub[0]), int(sub[1]))])) <= 1e-13 * scale
    trun_err = 1.0000000036274937e-15
    r0 = ctx.get_truncation_operator(side, gs.vec, cfg.kept_min, cfg.sweeps[0], trun_err)
    r1 = ctx.truncation_from_density(den, cfg.kept_min, cfg.sweeps[0], trun_err)
    assert r1["num_state"] == r0["num_state"] and r1["err"] == r0["err"] and r1["entropy"] == r0["entropy"]
    assert np.array_equal(r1["spectrum"][:den.dim], r0["spectrum"][:den.dim])
    assert all(np.array_equal(a, b) for a, b in zip(r1["trun"].mats, r0["trun"].mats))
    rng = np.random.default_rng(7)
    psi2 = rng.standard_normal(gs.dim) + 1j * rng.standard_normal(gs.dim)
    den2 = ctx.get_density_matrix(side, [gs.vec, psi2])
    w2 = type(gs)(gs.sys_len, gs.env_len, gs.secs, psi2)
    for k, (sub, m) in enumerate(zip(den2.subs, den2.mats)):
        a, b = gs.sector(k), w2.sector(k)
        want = (a @ a.conj().T + b @ b.conj().T) / 2 if side == 0 else (a.conj().T @ a + b.conj().T @ b) / 2
        assert np.max(np.abs(m - want)) <= 1e-12 * max(np.max(np.abs(want)), 1.0)


@pytest.mark.gpu
def test_renormalization_matches_oracle(captured):
    cfg, cap, ctx = captured
    side = 0 if cap["sys_side"] else 1
    pre = cap["sys"] if side == 0 else cap["env"]
    sys_len, env_len = cap["sys"].len, cap["env"].len
    mshift = 0 if side == 0 else (sys_len + 1)
    grown = ctx.get_hamiltonian(side, pre, cap["grow_basis"], cap["trun"], sys_len, env_len, mshift)
    ref = cap["grown"]
    assert grown.len == ref.len and len(grown.ops) == len(ref.ops)
    scale = max(np.max(np.abs(m)) for m in ref.ham.mats)
    for a, b in zip(grown.ham.mats, ref.ham.mats):
        assert np.max(np.abs(a - b)) <= 1e-12 * scale
    for oa, ob in zip(grown.ops, ref.ops):
        for ba, bb in zip(oa, ob):
            assert (ba.subs == bb.subs).all()
            for a, b in zip(ba.mats, bb.mats):
                assert np.max(np.abs(a - b), initial=0.0) <= 1e-12 * max(scale, 1.0)


@pytest.mark.gpu
def test_wave_transform_matches_oracle(captured):
    _, cap, ctx = captured
    if not cap["has_wt"]:
        pytest.skip("step starts from a random state")
    new = ctx.wave_trans(0 if cap["wt_lr"] else 1, cap["wt_sys_bs"], cap["wt_env_bs"], cap["wt_sys_trun"],
                         cap["wt_env_trun"], cap["wt_old"], cap["wt_new"])
    assert rel(new.vec, cap["wt_new"].vec) <= 1e-12


@pytest.mark.gpu
def test_full_sweep_matches_oracle():
    """Whole Get_Ground_State on the device vs the oracle: YC4x4, t2/J2 on, m=60."""
    cfg = orc.RunConfig(Nx=4, Ny=4, t1=1.0, t2=0.3, J1=0.4, J2=0.036, kept_min=60, kept_warm=60, sweeps=[60, 80],
                        lanzero=1e-10)
    ref = orc.Oracle(cfg).run()
    ctx = Context(4, 4, 1.0, 0.3, 0.4, 0.036)
    got = ctx.get_ground_state(60, 60, [60, 80], lanzero=1e-10, seed=1)
    ctx.close()
    assert len(got) == len(ref)
    for g, r in zip(got, ref):
        assert (g["sys_len"], g["env_len"]) == (r["sys_len"], r["env_len"])
        assert abs(g["e0"] - r["e0"]) <= 1e-10 * abs(r["e0"])
        assert g["num_state"] == r["num_state"]
