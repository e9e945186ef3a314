"""Comoving coordinates (supercomoving): the expansion factor's time
integration (cosmostart, compcosmo with rungekutta, cosmostep, updatetime's
comoving branch with timestepiteration; cosmology.f90, timestep.f90), the
comoving units (compunits, units.f90) and the expansion terms (expansion,
cosmology.f90:53-72) in the hand oracle, against the reference's Fortran
translated to C, bit for bit; and the library's host forms of the same
scalar routines (evora_cosmostart ... evora_updatetime_cosmo, evora_compunits)
against the oracle.  No GPU needed."""
import ctypes

import numpy as np
import pytest

import evora_b200 as ev
from evora_b200 import _native
from evora_b200.hydro import DropIn
from oracle import ref_oracle
from oracle.oracle import TIME_FIELDS, Oracle, make_params
from oracle.ref_oracle import RefOracle
from helpers import random_q

needs_ref = pytest.mark.skipif(not ref_oracle.available(), reason="translated reference not built")

COSMO = [
    dict(omega0=1.0, lambda0=0.0, zstart=10.0, zend=9.0),
    dict(omega0=0.3, lambda0=0.7, hubble0=70.0, box=20.0, zstart=30.0, zend=25.0, c_cosmo=0.05),
    dict(omega0=0.3, lambda0=0.7, hubble0=70.0, box=5.0, zstart=4.0, zend=0.0),
]


def cparams(cfg, **kw):
    return make_params(supercomoving=1, **cfg, **kw)


@needs_ref
@pytest.mark.parametrize("cfg", COSMO)
def test_start_and_units_match_reference_bitwise(cfg):
    o, r = Oracle(cparams(cfg)), RefOracle(cparams(cfg))
    np.testing.assert_array_equal(o.time(), r.time())
    np.testing.assert_array_equal(o.units(), r.units())
    s = o.time()
    assert s[2] == 1.0 / (1.0 + cfg["zstart"]) and s[6] == cfg["zstart"]


@needs_ref
@pytest.mark.parametrize("cfg", COSMO)
def test_time_scalars_match_reference_bitwise(cfg):
    """cosmostep, compcosmo, updatetime and compunits along 40 steps of
    varying hydro dt, with dumps on the way and the last step shortened onto
    zend."""
    zs, ze = cfg["zstart"], cfg["zend"]
    dumps = list(np.linspace(zs, ze, 5)[1:-1])
    o, r = Oracle(cparams(cfg, dump_redshift=dumps)), RefOracle(cparams(cfg, dump_redshift=dumps))
    rng = np.random.default_rng(3)
    s_o, s_r = o.time(), r.time()
    go, k4, ndump = True, 1, 0
    for _ in range(400):
        dt_hydro = float(rng.uniform(0.2, 2.0)) * 10.0 ** rng.uniform(-3, 0)
        s_o[1] = s_r[1] = dt_hydro
        s_o = o.cosmostep(s_o)
        s_r, st = r.cosmostep(s_r)
        assert st == 0
        s_o = o.compcosmo(s_o)
        s_r, st = r.compcosmo(s_r)
        go_o, dump_o, s_o = o.updatetime_cosmo(go, s_o, k4)
        go_r, dump_r, s_r, st = r.updatetime_cosmo(go, s_r, k4)
        assert st == 0 and (go_o, dump_o) == (go_r, dump_r)
        np.testing.assert_array_equal(s_o, s_r)
        o.settime(s_o)
        assert r.settime(s_r) == 0
        np.testing.assert_array_equal(o.units(), r.units())
        if dump_o:
            ndump += 1
            assert abs(s_o[6] - dumps[k4 - 1]) < 1e-9 * (1 + abs(dumps[k4 - 1]))
            k4 += 1
        go = go_o
        if not go:
            break
    assert not go, "zend not reached"
    assert abs(s_o[6] - ze) < 1e-9 * (1 + ze)
    # a step lands on one event at most: zend first, then the next dump
    # (timestep.f90:154-161), so a long step can pass a dump redshift by
    assert 1 <= ndump <= len(dumps)
    assert o.error() == 0


@needs_ref
@pytest.mark.parametrize("cfg", COSMO)
def test_peebles_matches_reference_bitwise(cfg):
    """peebles (cosmology.f90:76-97, with trapezoid and peeblesint): oracle
    against the translation, and the library's evora_peebles against the
    oracle, at the start and at a later a."""
    o, r = Oracle(cparams(cfg)), RefOracle(cparams(cfg))
    drop = DropIn(_lib_params(cfg))
    for a in (1.0 / (1.0 + cfg["zstart"]), 0.05):
        s = o.time()
        s[2] = a
        f_o = o.peebles(s)
        f_r, st = r.peebles(s)
        assert st == 0 and f_o == f_r
        assert drop.peebles(dict(zip(TIME_FIELDS, s))) == f_o
        if cfg["lambda0"] == 0.0:
            assert abs(f_o - 1.0) < 1e-4          # Einstein-de Sitter: D ~ a


@needs_ref
@pytest.mark.parametrize("cfg", COSMO[:2])
def test_expansion_matches_reference_bitwise(cfg):
    for de in (0, 1):
        p = cparams(cfg, nx=12, ny=10, nz=8, dualenergy=de, de_thresh=0.3)
        o, r = Oracle(p), RefOracle(p)
        q = random_q(o, np.random.default_rng(5), pres=(0.3, 3.0))
        if de:
            q[..., 5] *= 1.02
        s = o.time()
        s[1], s[5] = 0.37, 0.021          # dt, expand
        q_o, q_r = q.copy(), q.copy()
        o.expansion(q_o, s)
        assert r.expansion(q_r, s) == 0
        np.testing.assert_array_equal(q_o, q_r)
        assert not np.array_equal(q_o[..., 4], q[..., 4])


RUNS = [
    dict(nx=16, ny=14, nz=12, boundtype=2),
    dict(nx=24, ny=20, nz=1, boundtype=3, tempfloor=1, temp_fl=0.5),
    # simplekappa's flux (kappa = 1/(g-1) on T = p/rho temp0) against the
    # kappa0 T^2.5 time-step limit is stable only where temp0 is small: a
    # tiny box (the reference's own combination, unchanged)
    dict(nx=12, ny=10, nz=8, boundtype=2, conduction=1, simplekappa=1, box=1e-5),
    dict(nx=12, ny=10, nz=8, boundtype=1, dualenergy=1, de_thresh=0.3, atomic=1),
    dict(nx=64, ny=1, nz=1, boundtype=1, jeansfloor=1, c_jeans=0.05),
]


@needs_ref
@pytest.mark.parametrize("cfg", RUNS, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
def test_comoving_runs_match_reference_bitwise(cfg):
    """The loop of main.f90:109-203 with supercomoving: per step the time
    scalars after updatetime and the dumps raised, and the state at the end
    (zend reached), bit for bit."""
    cos = dict(omega0=1.0, lambda0=0.0, zstart=10.0, zend=9.6, dump_redshift=[9.9, 9.75])
    p = make_params(supercomoving=1, g=5 / 3 if cfg.get("atomic") else 1.4, cfl=0.4, **cos, **cfg)
    o, r = Oracle(p), RefOracle(p)
    q = random_q(o, np.random.default_rng(17), pres=(0.3, 3.0))
    q_o, q_r = q.copy(), q.copy()
    a = o.run(q_o, 400, trace=True)
    b = r.run(q_r, 400, trace=True)
    assert a["status"] == 0 and b["stopped"] == 0
    assert a["steps"] == b["steps"] and not a["go"] and not b["go"]
    np.testing.assert_array_equal(a["trace"], b["trace"])
    np.testing.assert_array_equal(q_o, q_r)
    dumps = a["trace"][:, 7]
    assert list(dumps[dumps > 0]) == [1.0, 2.0]
    assert abs(a["trace"][-1, 6] - 9.6) < 1e-9


# ----------------------------------------------- the library's host forms --
def _lib_params(cfg, **kw):
    return ev.default_params(supercomoving=1, **cfg, **kw)


def _as_array(d):
    return np.array([d[k] for k in TIME_FIELDS])


@pytest.mark.parametrize("cfg", COSMO)
def test_library_time_routines_match_oracle_bitwise(cfg):
    zs, ze = cfg["zstart"], cfg["zend"]
    dumps = list(np.linspace(zs, ze, 4)[1:-1])
    P = _lib_params(cfg, dump_redshift=dumps)
    drop = DropIn(P)
    drop._activate()
    o = Oracle(cparams(cfg, dump_redshift=dumps))
    s_l = drop.cosmostart()
    s_o = o.time()
    np.testing.assert_array_equal(_as_array(s_l), s_o)
    rng = np.random.default_rng(4)
    go, k4 = True, 1
    for _ in range(400):
        dt_hydro = float(rng.uniform(0.2, 2.0)) * 10.0 ** rng.uniform(-3, 0)
        s_l["dt"] = dt_hydro
        s_o[1] = dt_hydro
        s_l = drop.compcosmo(drop.cosmostep(s_l))
        s_o = o.compcosmo(o.cosmostep(s_o))
        go_l, dump_l, s_l = drop.updatetime_cosmo(go, s_l, k4)
        go_o, dump_o, s_o = o.updatetime_cosmo(go, s_o, k4)
        assert (go_l, dump_l) == (go_o, dump_o)
        np.testing.assert_array_equal(_as_array(s_l), s_o)
        if dump_l:
            k4 += 1
        go = go_l
        if not go:
            break
    assert not go and 2 <= k4 <= len(dumps) + 1


@pytest.mark.parametrize("cfg", COSMO)
def test_library_compunits_match_oracle_bitwise(cfg):
    """evora_compunits (the units file's values) at the start and after a
    few steps of a, against the oracle's compunits: temp0, kappa0."""
    P = _lib_params(cfg)
    o = Oracle(cparams(cfg))
    u = _native.EvoraUnits()
    assert _native.lib().evora_compunits(ctypes.byref(P), None, ctypes.byref(u)) == 0
    temp0, temp0inv, kappa0 = o.units()
    assert (u.temp0, u.kappa0) == (temp0, kappa0)
    assert u.cosmo == 1.0 / (1.0 + cfg["zstart"]) and u.redshift == cfg["zstart"]
    s = o.time()
    for dt in (0.01, 0.05, 0.2):
        s[1] = dt
        s = o.compcosmo(s)
        o.settime(s)
        t = _native.EvoraTime(*s)
        assert _native.lib().evora_compunits(ctypes.byref(P), ctypes.byref(t), ctypes.byref(u)) == 0
        assert (u.temp0, u.kappa0) == tuple(o.units()[[0, 2]])
        assert (u.cosmo, u.redshift) == (s[2], s[6])


def test_noncomoving_units_unchanged():
    """Without supercomoving compunits keeps the unit bases (cosmo = 1)."""
    P = ev.default_params(g=5 / 3)
    u1, u2 = _native.EvoraUnits(), _native.EvoraUnits()
    _native.lib().evora_units_noncomoving(0.0, P.g, 1.0, ctypes.byref(u1))
    assert _native.lib().evora_compunits(ctypes.byref(P), None, ctypes.byref(u2)) == 0
    for k in _native.EvoraUnits.NAMES:
        assert getattr(u1, k) == getattr(u2, k), k
