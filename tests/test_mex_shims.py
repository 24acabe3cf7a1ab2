"""The C MEX shims under mex/, built against a MEX API stand-in (tests/mexsim) and called
with MATLAB-shaped arguments.

CPU tests check that every shim builds and rejects bad calls before touching the GPU; GPU
tests check that each shim returns exactly what the C ABI returns for the same call.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "mexsim"))
import mexsim  # noqa: E402

from swd_b200 import configs  # noqa: E402

SHIMS = ["eigen_staggerfd_single", "eigen_staggerfd_double", "eigen_e2drtm_single", "eigen_e2drtm_double",
         "RTrAD", "RTlAD", "RTr", "RTl", "LHDispPick", "ADWDgrad_1", "ADWDgrad_norm", "ADWDgradlimband",
         "weight_data_muti3", "norm_trace", "fk_filter", "eigen_staggerfd_single_batch", "eigen_e2drtm_single_batch",
         "field/LHDispPick", "field/ADWDgrad_1"]


@pytest.fixture(scope="module")
def shim(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("mex"))
    cache = {}

    def get(name):
        if name not in cache:
            cache[name] = mexsim.Shim(name, d)
        return cache[name]
    return get


@pytest.mark.parametrize("name", SHIMS)
def test_shim_builds_and_checks_argument_count(shim, name):
    with pytest.raises(mexsim.MexError, match="swd:nrhs"):
        shim(name)(1, 1.0, 2.0)  # nlhs 1, two inputs: no shim takes two


def _fd_args(O, single=True, adjoint=False):
    s = configs.tiny(nt=400)
    inp = O.fd_inputs(s.nbc, s.nt, s.dtx, s.dx, s.dt, int(s.sx[1]), 1, s.gx, np.ones(s.ng), s.vp, s.vs,
                      source_type="w", in_wf=s.nt_wf, single=single, adjoint=adjoint)
    return s, inp


def test_fd_shims_reject_bad_classes_and_sizes(O, shim):
    s, inp = _fd_args(O)
    f = shim("eigen_staggerfd_single")
    w = s.source().astype(np.float32)
    args = [inp.iv, inp.temp, inp.ca, inp.cl, inp.cm, inp.cm1, inp.b, inp.b1, w]
    bad = list(args)
    bad[2] = inp.ca.astype(np.float64)
    with pytest.raises(mexsim.MexError, match="ca must be a real single"):
        f(3, *bad)
    bad = list(args)
    bad[3] = inp.cl[:, :5]
    with pytest.raises(mexsim.MexError, match="cl has"):
        f(3, *bad)
    bad = list(args)
    bad[8] = w[:10]
    with pytest.raises(mexsim.MexError, match="s has 10 elements"):
        f(3, *bad)
    iv = inp.iv.copy()
    iv[11] = 24  # fd_order 24: accepted by the reference, not built here
    with pytest.raises(mexsim.MexError, match="fd_order 24"):
        f(3, iv, *args[1:])


def test_radon_shims_check_np_and_adwdgrad_needs_shim_structs(shim):
    s = configs.tiny(nt=400)
    seis = np.zeros((s.nt, s.ng))
    with pytest.raises(mexsim.MexError, match="np"):
        shim("RTrAD")(3, seis, 1, s.df, s.dt, 5, s.vmin, s.vmax, s.fmin, s.fmax, s.nt, s.ng, s.ds, s.offset, s.m,
                      s.M)
    npair = s.npair
    with pytest.raises(mexsim.MexError, match="swd_params"):
        shim("ADWDgrad_1")(1, s.nt, s.ng, s.ns, npair, 2, s.w, s.m, s.M, 1e4, np.ones(npair), np.ones(npair),
                           np.ones((701, npair)), {"mm": np.zeros((3, 3))}, {"mm": np.zeros((3, 3))})


@pytest.mark.parametrize("name,nrhs", [("eigen_staggerfd_single_batch", 9), ("eigen_e2drtm_single_batch", 13)])
def test_batch_shims_check_their_cell_arrays(shim, name, nrhs):
    f = shim(name)
    with pytest.raises(mexsim.MexError, match="cell array"):
        f(1, *([np.zeros(3, np.float32)] * nrhs))
    with pytest.raises(mexsim.MexError, match="entries"):
        f(1, *([[np.zeros(3, np.float32)]] * (nrhs - 1)), [])


@pytest.mark.gpu
def test_batch_shims_match_the_single_shims(O, shim):
    """Two jobs on different grids in one eigen_staggerfd_single_batch call (cell arrays in and
    out) give what two eigen_staggerfd_single calls give; likewise eigen_e2drtm_single_batch
    against eigen_e2drtm_single on those jobs' wavefields."""
    import dataclasses

    from swd_b200 import configs
    cases = [configs.tiny(nt=400), dataclasses.replace(configs.plain_c1(), nt=800, nt_wf=10)]
    args, refs = [[] for _ in range(9)], []
    for s in cases:
        inp = O.fd_inputs(s.nbc, s.nt, s.dtx, s.dx, s.dt, int(s.sx[1]), 1, s.gx, np.ones(s.ng), s.vp, s.vs,
                          in_wf=s.nt_wf)
        w = s.source().astype(np.float32)
        one = (inp.iv, inp.temp, inp.ca, inp.cl, inp.cm, inp.cm1, inp.b, inp.b1, w)
        for k in range(9):
            args[k].append(one[k])
        refs.append(shim("eigen_staggerfd_single")(3, *one))
    su, sw, www = shim("eigen_staggerfd_single_batch")(3, *args)
    for j, (ru, rw, rwww) in enumerate(refs):
        assert np.array_equal(su[j], ru) and np.array_equal(sw[j], rw), j
        for k in ("fux", "fuz", "bwx", "bwz"):
            assert np.array_equal(www[j][k], rwww[k]), (j, k)
    rng = np.random.default_rng(2)
    aargs, arefs = [[] for _ in range(13)], []
    for s, (_, rw, rwww) in zip(cases, refs):
        ainp = O.fd_inputs(s.nbc, s.nt, s.dtx, s.dx, s.dt, int(s.sx[1]), 1, s.gx, np.ones(s.ng), s.vp, s.vs,
                           in_wf=s.nt_wf, adjoint=True)
        res = (rng.standard_normal(rw.shape) * 1e-3).astype(np.float32)
        one = (ainp.iv, ainp.temp, ainp.ca, ainp.cl, ainp.cm, ainp.cm1, ainp.b, ainp.b1, res, rwww["fux"],
               rwww["fuz"], rwww["bwx"], rwww["bwz"])
        for k in range(13):
            aargs[k].append(one[k])
        arefs.append(shim("eigen_e2drtm_single")(3, *one))
    got = shim("eigen_e2drtm_single_batch")(3, *aargs)
    for j, want in enumerate(arefs):
        for k in range(3):
            assert got[k][j].dtype == np.float32 and np.abs(want[k]).max() > 0, (j, k)
            assert np.array_equal(got[k][j], want[k]), (j, k)


@pytest.mark.gpu
@pytest.mark.parametrize("single", [True, False])
def test_fd_shims_match_the_c_abi(O, shim, single):
    import swd_b200 as S
    s, inp = _fd_args(O, single)
    dt = np.float32 if single else np.float64
    w = s.source().astype(dt)
    name = "single" if single else "double"
    su, sw, www = shim("eigen_staggerfd_" + name)(3, inp.iv, inp.temp, inp.ca, inp.cl, inp.cm, inp.cm1, inp.b, inp.b1,
                                                 w)
    ref = getattr(S, "eigen_staggerfd_" + name)(inp.iv, inp.temp, inp.ca, inp.cl, inp.cm, inp.cm1, inp.b, inp.b1, w)
    assert su.dtype == dt and su.shape == (s.nt, s.ng)
    assert np.array_equal(su, ref[0]) and np.array_equal(sw, ref[1])
    for k in ("fux", "fuz", "bwx", "bwz"):
        assert www[k].shape == ref[2][k].shape and np.array_equal(www[k], ref[2][k]), k
    # two outputs: no snapshots are kept, seismograms unchanged
    su2, sw2 = shim("eigen_staggerfd_" + name)(2, inp.iv, inp.temp, inp.ca, inp.cl, inp.cm, inp.cm1, inp.b, inp.b1, w)
    assert np.array_equal(sw2, sw)
    _, ainp = _fd_args(O, single, adjoint=True)
    res = (np.random.default_rng(1).standard_normal(sw.shape) * 1e-3).astype(dt)
    got = shim("eigen_e2drtm_" + name)(3, ainp.iv, ainp.temp, ainp.ca, ainp.cl, ainp.cm, ainp.cm1, ainp.b, ainp.b1,
                                       res, www["fux"], www["fuz"], www["bwx"], www["bwz"])
    want = getattr(S, "eigen_e2drtm_" + name)(ainp.iv, ainp.temp, ainp.ca, ainp.cl, ainp.cm, ainp.cm1, ainp.b,
                                               ainp.b1, res, www["fux"], www["fuz"], www["bwx"], www["bwz"])
    for g, r in zip(got, want):
        assert g.dtype == dt and np.abs(r).max() > 0 and np.array_equal(g, r)


@pytest.mark.gpu
def test_spectrum_shims_match_the_c_abi(O, shim):
    from swd_b200 import spectrum as SP
    s = configs.tiny(nt=400, ns=5)
    is_ = 3
    inp = O.fd_inputs(s.nbc, s.nt, s.dtx, s.dx, s.dt, int(s.sx[is_ - 1]), 1, s.gx, np.ones(s.ng), s.vp, s.vs,
                      source_type="w", in_wf=s.nt_wf)
    _, sw, _ = O.mex_staggerfd(inp, s.source(), want_wf=False)
    seis = sw.astype(np.float64)
    vmax = s.vmin + 60  # 1 m/s steps as the reference's pp = 1./(vmin:vmax)'
    npv = int(vmax - s.vmin) + 1
    args = (is_, s.df, s.dt, npv, s.vmin, vmax, s.fmin, s.fmax, s.nt, s.ng, s.ds, s.offset, s.m, s.M)
    out = {}
    for side, name in ((0, "RTrAD"), (1, "RTlAD")):
        ml, n, sfb = shim(name)(3, seis, *args)
        rml, rn, rs = getattr(SP, name)(seis, *args)
        assert np.array_equal(ml, rml) and n == rn
        raw = "mlr" if side == 0 else "mll"
        pos = "uxtposr" if side == 0 else "uxtposl"
        assert np.array_equal(sfb[raw], rs[raw]) and np.array_equal(sfb["mm"], rs["mm"])
        assert np.array_equal(sfb[pos].ravel(), rs[pos]) and sfb["lf"] == rs["lf"] and sfb["nf"] == rs["nf"]
        assert sfb["ccn"] == rs["ccn"]
        np.testing.assert_allclose(sfb["ll0"], rs["ll0"], rtol=1e-15)
        ml2, n2 = shim(name[:3])(2, seis, *args)
        assert np.array_equal(ml2, ml) and n2 == n
        out[side] = (ml, sfb, rs)
    npair = out[0][0].shape[1]
    cr0 = np.full(npair, s.vmin + 20.0)
    res, cr = shim("LHDispPick")(2, out[0][0], s.vmin, cr0, 1, s.ini)
    rres, rcr = SP.LHDispPick(out[0][0], s.vmin, cr0, 1, s.ini)
    assert cr.shape == (npair, 1) and np.array_equal(cr.ravel(), rcr) and res == rres
    space = np.repeat(np.arange(1.0, npv + 1)[:, None], npair, 1)
    gr, gl = rcr - cr0, np.linspace(-3, 3, npair)
    a = shim("ADWDgrad_1")(1, s.nt, s.ng, s.ns, npair, is_, s.w, s.m, s.M, s.soft_arg_norm, gr, gl, space,
                           out[0][1], out[1][1])[0]
    ra = SP.ADWDgrad_1(s.nt, s.ng, s.ns, npair, is_, s.w, s.m, s.M, s.soft_arg_norm, gr, gl, space, out[0][2],
                       out[1][2])
    assert np.abs(ra).max() > 0 and np.array_equal(a, ra)
    # ADWDgrad_norm: the structs also carry the picks minus vmin (SWD.m:178, :184)
    cr_r, cr_l = rcr - s.vmin, np.linspace(2.0, npv - 2.0, npair)
    sr, sl = dict(out[0][1], cr_r=cr_r), dict(out[1][1], cr_l=cr_l)
    an = shim("ADWDgrad_norm")(1, s.nt, s.ng, s.ns, npair, is_, s.w, s.m, s.M, s.soft_arg_norm, gr, gl, space,
                               sr, sl)[0]
    ran = SP.ADWDgrad_norm(s.nt, s.ng, s.ns, npair, is_, s.w, s.m, s.M, s.soft_arg_norm, gr, gl, space,
                           dict(out[0][2], cr_r=cr_r), dict(out[1][2], cr_l=cr_l))
    assert np.abs(ran).max() > 0 and np.array_equal(an, ran)
    with pytest.raises(mexsim.MexError, match="cr_r"):
        shim("ADWDgrad_norm")(1, s.nt, s.ng, s.ns, npair, is_, s.w, s.m, s.M, s.soft_arg_norm, gr, gl, space,
                              out[0][1], sl)


@pytest.mark.gpu
def test_wd_shim_matches_the_c_abi(O, shim):
    from swd_b200 import spectrum as SP
    rng = np.random.default_rng(4)
    nt, ng, dt, df, fmin, fmax = 300, 40, 1e-3, 2.0, 10.0, 40.0
    ind, npair = 6, 16
    refsx = np.floor(1 + 3 * np.arange(12)) + 1
    pred = rng.standard_normal((nt, ng)).astype(np.float32)  # SWD_single.m's single seismo_v
    cr0, crp = 300 + 50 * rng.random(npair), 300 + 50 * rng.random(npair)
    args = (5, dt, df, 12, 0.5, 0, 3, 3.0, 0, 12, refsx, npair + 2 * ind, fmin, fmax, cr0, cr0[::-1].copy(), crp,
            crp[::-1].copy(), float(ind))
    got = shim("weight_data_muti3")(1, np.zeros((nt, ng)), pred, *args)[0]
    want = SP.weight_data_muti3(None, pred.astype(np.float64), *args)
    assert np.abs(want).max() > 0 and np.array_equal(got, want)
    with pytest.raises(mexsim.MexError, match="picks"):
        shim("weight_data_muti3")(1, np.zeros((nt, ng)), pred, *args[:14], cr0[:5], *args[15:])
