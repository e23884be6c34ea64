"""Parse the oracle's captured superblock (oracle/oracle_driver.cpp, orc_capture_serialize)."""
from tsc_tri_t1t2j1j2_b200.layout import Basis, Block, Cursor, Model, Wave


def parse_oracle_capture(ints, data):
    c = Cursor(ints, data)
    valid, sys_side, iters, num_state, nxc, has_wt, wt_lr, sn, en, gn = (int(x) for x in c.take(10))
    e0, err, ent, entm = (float(x.real) for x in c.cdata(4))
    cap = dict(sys_side=sys_side, iters=iters, num_state=num_state, nxc=nxc, has_wt=has_wt, wt_lr=wt_lr,
               e0=e0, err=err, ent=ent, ent_mult=entm)
    cap["sys"] = Model.read(c)
    cap["env"] = Model.read(c)
    cap["sys_bs"] = Basis.read(c)
    cap["env_bs"] = Basis.read(c)
    cap["psi0"] = Wave.read(c)
    cap["hpsi"] = Wave.read(c)
    cap["gs"] = Wave.read(c)
    cap["den"] = Block.read(c)
    cap["trun"] = Block.read(c)
    cap["grow_basis"] = Basis.read(c)
    cap["grown"] = Model.read(c)
    nspec = c.one()
    cap["spectrum"] = c.cdata(nspec).real.copy()
    if has_wt:
        cap["wt_sys_bs"] = Basis.read(c)
        cap["wt_env_bs"] = Basis.read(c)
        cap["wt_sys_trun"] = Block.read(c)
        cap["wt_env_trun"] = Block.read(c)
        cap["wt_old"] = Wave.read(c)
        cap["wt_new"] = Wave.read(c)
    return cap
