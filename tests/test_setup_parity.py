"""CPU tests: the product's host setup against the oracle (bit-exact), the
C-ABI symbol table, and the input reader.  No GPU needed."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from openswpc_b200 import _lib
from openswpc_b200.params import Layer, Params, Source, Station, dc_source, params_from_ini
from openswpc_b200.swpc3d import Medium, grid_struct, source_grid, station_grid
from oracle.oracle import Oracle3D, load as oload
from tests.models import LAYERS, small3d, vonkarman_xi

ROOT = Path(__file__).resolve().parents[1]


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32 if a.dtype == np.float32 else np.uint64)


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    declared = set()
    for h in (ROOT / "include").glob("*.h"):
        txt = h.read_text()
        declared |= set(re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(swpc_\w+)\s*\(", txt, flags=re.M))
    assert len(declared) > 30
    missing = [s for s in sorted(declared) if not hasattr(lib, s)]
    assert not missing, missing
    assert set(_lib.EXPORTS) <= declared | set(_lib.EXPORTS)


@pytest.mark.parametrize("with_xi", [False, True])
def test_medium_setup_bit_exact(with_xi):
    p = small3d()
    xi = vonkarman_xi((p.ny + 6, p.nx + 6, p.nz + 6)) if with_xi else None
    m = Medium(p, xi)
    o = Oracle3D(p, xi)
    for f in ("rho", "lam", "mu", "taup", "taus", "bx", "by", "bz", "muyz", "muxz", "muxy"):
        assert np.array_equal(bits(getattr(m, f)), bits(o.array("f" + f))), f
    for f in ("kfs", "kob", "kfs_top", "kfs_bot", "kob_top", "kob_bot", "kbeg_a"):
        assert np.array_equal(getattr(m, f), o.array(f)), f
    sc = o.scalars()
    assert np.float32(sc["zeta"]) == np.float32(m.zeta)
    assert np.float32(sc["vmin"]) == np.float32(m.vmin) and np.float32(sc["vmax"]) == np.float32(m.vmax)
    assert np.array_equal(m.ts, np.array([sc["ts1"], sc["ts2"], sc["ts3"]], np.float32))


def test_free_surface_maps_locate_air_solid_boundary():
    p = small3d()
    m = Medium(p)
    # zbeg = -3 dz: cells k = 1..3 are air, k = 4 is the first solid cell
    assert (m.kfs[2:-3, 2:-3] == 3).all() and (m.kob[2:-3, 2:-3] == 3).all()
    assert (m.kfs_top[3:-3, 3:-3] == 1).all() and (m.kfs_bot[3:-3, 3:-3] == 5).all()


def test_source_and_station_maps_bit_exact():
    p = small3d(sources=[dc_source(0.3, -0.7, 6.1, 0.0, 1.0, 1e16, 30, 60, 90),
                         Source(2.2, 1.1, 4.0, 0.2, 1.5, mo=3e15, mxx=1, myy=1, mzz=1),
                         Source(-9.9, -8.9, 0.1, 0.0, 1.0, mo=1e15, mxy=1.0)])
    sg = source_grid(p)
    o = Oracle3D(p)
    d = o.dims()
    n = d["nsrc"]
    isrc = np.ctypeslib.as_array(C.cast(o.lib.o3d_ptr(o.o, 98), C.POINTER(C.c_int)), (n,))
    jsrc = np.ctypeslib.as_array(C.cast(o.lib.o3d_ptr(o.o, 99), C.POINTER(C.c_int)), (n,))
    ksrc = np.ctypeslib.as_array(C.cast(o.lib.o3d_ptr(o.o, 100), C.POINTER(C.c_int)), (n,))
    assert np.array_equal(sg.isrc, isrc) and np.array_equal(sg.jsrc, jsrc) and np.array_equal(sg.ksrc, ksrc)
    sc = o.scalars()
    assert np.float32(sc["M0"]) == np.float32(sg.M0) and np.float32(sc["fcut"]) == np.float32(sg.fcut)
    m = Medium(p)
    ist, jst, kst = station_grid(p, m.kfs, m.kob)
    assert np.array_equal(ist, o.ist) and np.array_equal(jst, o.jst) and np.array_equal(kst, o.kst)


def test_damping_profiles_bit_exact():
    p = small3d()
    lib = _lib.load()
    g = grid_struct(p)
    prof = {k: np.zeros((n, 4), np.float32) for k, n in
            (("gxc", p.nx), ("gxe", p.nx), ("gyc", p.ny), ("gye", p.ny), ("gzc", p.nz), ("gze", p.nz))}
    fcut = np.float32(1.0)
    lib.swpc_damping_profiles(C.byref(g), float(fcut), *[_lib.fptr(prof[k]) for k in ("gxc", "gxe", "gyc", "gye",
                                                                                     "gzc", "gze")])
    o = Oracle3D(p)   # source trise = 1.0 -> fcut = 1.0
    for n, k in enumerate(("gxc", "gxe", "gyc", "gye", "gzc", "gze")):
        cnt = prof[k].size
        ref = np.ctypeslib.as_array(C.cast(o.lib.o3d_ptr(o.o, 80 + n), C.POINTER(C.c_float)), (cnt,))
        assert np.array_equal(bits(prof[k].ravel()), bits(ref)), k
    # the profile is the identity (g1 = 1, g2 = -1... no damping) in the interior
    assert np.allclose(prof["gxc"][p.na + 2, :2], [1.0 / 1.0, -1.0], atol=1e-6) or prof["gxc"][p.na + 2, 3] == 0


@pytest.mark.parametrize("stf", ["kupper", "boxcar", "triangle", "herrmann", "cosine", "texp"])
def test_moment_rate_functions_match(stf):
    lib = _lib.load()
    ol = oload()
    code = _lib.STF_CODES[stf]
    for t in np.linspace(-0.5, 3.5, 401, dtype=np.float32):
        a = lib.swpc_momentrate(float(t), code, 0.25, 2.0)
        b = ol.o3d_momentrate(float(t), code, 0.25, 2.0)
        assert np.float32(a) == np.float32(b)


def test_moment_rate_integrates_to_one():
    lib = _lib.load()
    for stf, code in _lib.STF_CODES.items():
        if stf == "scosine":
            continue
        t = np.arange(0, 40.0, 1e-3, dtype=np.float64)
        v = np.array([lib.swpc_momentrate(float(x), code, 0.5, 2.0) for x in t[::10]])
        integral = v.sum() * 1e-2
        assert abs(integral - 1.0) < 2e-2, (stf, integral)


def test_sdr2moment_is_double_couple():
    lib = _lib.load()
    m6 = (C.c_float * 6)()
    for sdr in ((30, 60, 90), (0, 90, 0), (123, 45, -60)):
        lib.swpc_sdr2moment(*sdr, m6)
        m = np.array([[m6[0], m6[5], m6[4]], [m6[5], m6[1], m6[3]], [m6[4], m6[3], m6[2]]], np.float64)
        ev = np.sort(np.linalg.eigvalsh(m))
        assert np.allclose(ev, [-1, 0, 1], atol=1e-5)
        assert abs(np.trace(m)) < 1e-5


def test_grid_index_functions_match_oracle():
    lib = _lib.load()
    ol = oload()
    rng = np.random.default_rng(3)
    for x in rng.uniform(-50, 50, 500).astype(np.float32):
        for beg, d in ((-10.0, 0.1), (-96.0, 0.5), (-1.5, 0.25)):
            assert lib.swpc_x2i(float(x), beg, d) == ol.o3d_x2i(float(x), beg, d)
    for i in range(-3, 200):
        assert np.float32(lib.swpc_i2x(i, -10.0, 0.1)) == np.float32(ol.o3d_i2x(i, -10.0, 0.1))


def test_params_reader(tmp_path):
    (tmp_path / "lhm.dat").write_text("# d rho vp vs qp qs\n 0 2.7 5.5 3.2 300 150\n 5 2.8 6.0 3.5 500 250\n")
    (tmp_path / "src.dat").write_text("# x y z t0 tr mo mxx myy mzz myz mxz mxy\n0 0 6 0.1 2 1e16 1 1 1 0 0 0\n")
    (tmp_path / "st.xy").write_text("1.0 2.0 0.0 st01 fsb\n-3 4 0 st02 obb\n")
    (tmp_path / "input.inf").write_text(
        "title = 'x'  !! comment\n nx = 64\n ny = 48\n nz = 32\n nt = 10\n dx = 0.25\n dy=0.25\n dz = 0.25\n"
        " dt = 0.01\n na = 8\n zbeg = -1.0\n fn_lhm = 'lhm.dat'\n fn_stf = 'src.dat'\n stf_format='xym0ij'\n"
        " fn_stloc = 'st.xy'\n sw_wav_v = .true.\n ntdec_w = 2\n")
    p = params_from_ini(tmp_path / "input.inf")
    assert (p.nx, p.ny, p.nz, p.nt, p.na) == (64, 48, 32, 10, 8)
    assert p.dx == 0.25 and p.zbeg == -1.0 and p.ntdec_w == 2
    assert p.xbeg == -8.0 and p.ybeg == -6.0     # -nx/2*dx default
    assert len(p.layers) == 2 and len(p.sources) == 1 and len(p.stations) == 2
    assert p.sources[0].mo == 1e16 and p.stations[1].zsw == "obb"
    with pytest.raises(KeyError):
        params_from_ini(tmp_path / "input.inf", strict=True)


def test_oracle_fp32_close_to_fp64():
    """The restated scheme in FP32 stays within 1e-4 rel-L2 of the all-double
    build of the same scheme over a short run (sanity check of the oracle)."""
    p = small3d(nt=40)
    a = Oracle3D(p, variant="f32")
    b = Oracle3D(p, variant="f64")
    a.run(1, 40)
    b.run(1, 40)
    wa, wb = a.waveforms("v").astype(np.float64), b.waveforms("v").astype(np.float64)
    assert np.linalg.norm(wb) > 0
    assert np.linalg.norm(wa - wb) / np.linalg.norm(wb) < 1e-4
    va, vb = a.array("Vz").astype(np.float64), b.array("Vz")
    assert np.linalg.norm(va - vb) / np.linalg.norm(vb) < 1e-4


@pytest.mark.parametrize("kind", ["psv", "sh"])
def test_medium_setup_2d_bit_exact(kind):
    from openswpc_b200.swpc2d import Medium2D
    from oracle.oracle import Oracle2D
    from tests.models import small2d

    p = small2d(kind)
    m = Medium2D(p)
    o = Oracle2D(p, kind)
    for f in ("rho", "lam", "mu", "taup", "taus"):
        assert np.array_equal(bits(getattr(m, f)), bits(o.array("f" + f))), f
    for f in ("kfs", "kob", "kfs_top", "kfs_bot", "kob_top", "kob_bot", "kbeg_a"):
        assert np.array_equal(getattr(m, f), o.array(f)), f
    # the band follows the 3D formulation: [min(kfs)-2, max(kfs)+2]
    assert (m.kfs_top[5:-5] == 1).all() and (m.kfs_bot[5:-5] == 5).all()


@pytest.mark.parametrize("kind", ["psv", "sh"])
def test_oracle_2d_fp32_close_to_fp64(kind):
    from oracle.oracle import Oracle2D
    from tests.models import small2d

    p = small2d(kind, nt=60)
    a = Oracle2D(p, kind, "f32")
    b = Oracle2D(p, kind, "f64")
    a.run(1, 60)
    b.run(1, 60)
    wa, wb = a.waveforms("v").astype(np.float64), b.waveforms("v").astype(np.float64)
    assert np.linalg.norm(wb) > 0
    assert np.linalg.norm(wa - wb) / np.linalg.norm(wb) < 1e-4


def test_cerjan_profiles_match_oracle():
    """swpc_cerjan_profiles (absorb_c__setup, m_absorb_c.f90:27-103) against
    the oracle's sponge factors, bitwise; the free-surface side is 1."""
    import ctypes as C

    from openswpc_b200 import _lib
    from openswpc_b200.swpc3d import grid_struct
    from oracle.oracle import Oracle3D
    from tests.models import small3d

    p = small3d(nx=40, ny=36, nz=32, na=8, nt=2, abc_type="cerjan")
    lib = _lib.load()
    n = {"x": p.nx, "y": p.ny, "z": p.nz}
    names = ("gx_c", "gx_b", "gy_c", "gy_b", "gz_c", "gz_b")
    prof = {k: np.zeros(n[k[1]], np.float32) for k in names}
    lib.swpc_cerjan_profiles(C.byref(grid_struct(p)), *(_lib.fptr(prof[k]) for k in names))
    o = Oracle3D(p)
    for k in names:
        b = o.array(k)
        assert np.array_equal(prof[k].view(np.uint32), b.astype(np.float32).view(np.uint32)), k
    assert np.all(prof["gz_c"][:p.na] == 1.0) and prof["gz_c"][-1] < 1.0
    assert prof["gx_c"][0] < prof["gx_c"][p.na - 1] < 1.0 and prof["gx_c"][p.na] == 1.0


def test_cerjan_profiles_2d_match_oracle():
    """The 2D sponge factors (gy omitted) against the 2D oracle, bitwise."""
    from openswpc_b200 import _lib
    from openswpc_b200.swpc2d import grid2d
    from oracle.oracle import Oracle2D
    from tests.models import small2d

    p = small2d("psv", nt=2, abc_type="cerjan")
    lib = _lib.load()
    prof = {k: np.zeros(p.nx if k[1] == "x" else p.nz, np.float32) for k in ("gx_c", "gx_b", "gz_c", "gz_b")}
    lib.swpc_cerjan_profiles(C.byref(grid2d(p)), _lib.fptr(prof["gx_c"]), _lib.fptr(prof["gx_b"]), None, None,
                             _lib.fptr(prof["gz_c"]), _lib.fptr(prof["gz_b"]))
    o = Oracle2D(p, "psv")
    for k, v in prof.items():
        assert np.array_equal(v.view(np.uint32), o.array(k).astype(np.float32).view(np.uint32)), k


def test_stabilize_pml_matches_oracle():
    """stabilize_pml (m_medium.f90:219-222, stabilize_absorber :276-340): a
    thin low-velocity layer inside the absorber takes the medium above it and
    slow cells are raised to 0.4 vmax, bitwise as the oracle; the interior
    away from the absorber is untouched."""
    from openswpc_b200.swpc3d import Medium
    from tests.models import LAYERS, small3d

    # a 1 km low-velocity layer at 3 km depth, and a slow top layer
    layers = [Layer(0.0, 2.2, 2.4, 1.2, 100, 50), Layer(1.0, 2.7, 5.5, 3.2, 300, 150),
              Layer(3.0, 2.4, 3.0, 1.6, 100, 50), Layer(4.0, 2.7, 5.5, 3.2, 300, 150)] + LAYERS[1:]
    p = small3d(nx=40, ny=36, nz=32, na=8, nt=2, layers=layers, stabilize_pml=True)
    q = small3d(nx=40, ny=36, nz=32, na=8, nt=2, layers=layers)
    m, m0 = Medium(p), Medium(q)
    o = Oracle3D(p)
    for name in ("lam", "mu", "taup", "taus", "bx", "by", "bz", "muyz", "muxz", "muxy"):
        b = o.array(name).astype(np.float32)
        assert np.array_equal(getattr(m, name).view(np.uint32), b.view(np.uint32)), name
    assert not np.array_equal(m.mu, m0.mu)                     # the switch acted
    c = (slice(14, 26), slice(14, 30), slice(3, 20))           # columns away from the absorber
    assert np.array_equal(m.mu[c], m0.mu[c])


@pytest.mark.parametrize("kind", ["psv", "sh"])
def test_stabilize_pml_2d_matches_oracle(kind):
    """The 2D stabilize_absorber (src/swpc_psv/m_medium.f90:309-365), which
    fills the whole thin low-velocity layer, bitwise as the oracle."""
    from openswpc_b200.swpc2d import Medium2D
    from oracle.oracle import Oracle2D
    from tests.models import LAYERS, small2d

    layers = [Layer(0.0, 2.2, 2.4, 1.2, 100, 50), Layer(1.0, 2.7, 5.5, 3.2, 300, 150),
              Layer(3.0, 2.4, 3.0, 1.6, 100, 50), Layer(4.0, 2.7, 5.5, 3.2, 300, 150)] + LAYERS[1:]
    p = small2d(kind, nt=2, layers=layers, stabilize_pml=True)
    q = small2d(kind, nt=2, layers=layers)
    m, m0 = Medium2D(p), Medium2D(q)
    o = Oracle2D(p, kind)
    for name in ("rho", "lam", "mu", "taup", "taus"):
        b = o.array(name).astype(np.float32)
        assert np.array_equal(getattr(m, name).view(np.uint32), b.view(np.uint32)), name
    assert not np.array_equal(m.mu, m0.mu)


def test_sdr2moment_bit_exact_against_oracle():
    """The library's sdr2moment and the oracle's restatement agree bit for bit
    (m_fdtool.f90:307-336), so double couples enter both runs identically."""
    lib = _lib.load()
    ol = oload()
    rng = np.random.default_rng(11)
    sdrs = [(30, 60, 90), (0, 90, 0), (360, 90, 180), (-360, -90, -180), (123.4, 45.6, -60.7)]
    sdrs += [tuple(v) for v in np.stack([rng.uniform(-360, 360, 2000), rng.uniform(-90, 90, 2000),
                                         rng.uniform(-180, 180, 2000)], 1).astype(np.float32)]
    a, b = (C.c_float * 6)(), (C.c_float * 6)()
    for sdr in sdrs:
        lib.swpc_sdr2moment(*map(float, sdr), a)
        ol.o3d_sdr2moment(*map(float, sdr), b)
        assert np.array_equal(bits(np.array(a[:], np.float32)), bits(np.array(b[:], np.float32))), sdr


def test_dc_source_moment_is_formed_by_each_side():
    """A double couple carries strike/dip/rake; the product forms its tensor
    at source setup and the oracle with its own sdr2moment."""
    p = small3d(sources=[dc_source(0.3, -0.7, 6.1, 0.0, 1.0, 1e16, 30, 60, 90, phi=10.0)])
    s = p.sources[0]
    assert s.strike == np.float32(20.0) and s.mxx == 0.0
    sg = source_grid(p)
    ref = (C.c_float * 6)()
    oload().o3d_sdr2moment(20.0, 60.0, 90.0, ref)
    assert np.array_equal(bits(sg.m6[0]), bits(np.array(ref[:], np.float32)))


def _bd_params(custom: bool, two_d: bool = False):
    """Stations in every depth mode (dep fsb obb oba bd0-bd9), an unknown mode
    among them, and optionally boundary depths of the caller's own."""
    from tests.models import small2d

    modes = ["dep", "fsb", "obb", "oba"] + [f"bd{n}" for n in range(10)]
    rng = np.random.default_rng(21)
    p = small2d() if two_d else small3d()
    st = []
    for q, z in enumerate(modes * 2):
        x = float(rng.uniform(p.xbeg + (p.na + 2) * p.dx, p.xbeg + (p.nx - p.na - 2) * p.dx))
        y = 0.0 if two_d else float(rng.uniform(p.ybeg + (p.na + 2) * p.dy, p.ybeg + (p.ny - p.na - 2) * p.dy))
        st.append(Station(x, y, float(rng.uniform(0.5, 6.0)), f"b{q}", z))
    p.stations = st
    if custom:
        shape = (p.nx + 6, 10) if two_d else (p.ny + 6, p.nx + 6, 10)
        bd = rng.uniform(-1.0, 0.6 * p.nz * p.dz, shape).astype(np.float32)
        bd[..., 9] = 99.0     # below the model: clamped to kend - 1
        bd[..., 8] = -50.0    # above the model: clamped to kbeg + 1
        p.bddep = bd
    return p


@pytest.mark.parametrize("custom", [False, True])
def test_station_depth_modes_bit_exact(custom):
    """set_stinfo's depth modes, bd0-bd9 included (m_wav.f90:209-236): the
    station cells equal the oracle's, with vmodel_lhm's boundary depths
    (depth(1), then -9999) or the caller's."""
    p = _bd_params(custom)
    m = Medium(p)
    ist, jst, kst = station_grid(p, m.kfs, m.kob)
    o = Oracle3D(p)
    assert len(ist) == len(p.stations) == o.nst
    assert np.array_equal(ist, o.ist) and np.array_equal(jst, o.jst) and np.array_equal(kst, o.kst)
    # the boundary-depth stations did not all land on the 'dep' cell
    assert len(set(kst[4:14].tolist())) > (3 if custom else 1)


@pytest.mark.parametrize("custom", [False, True])
def test_station_depth_modes_bit_exact_2d(custom):
    """The same depth modes in the P-SV code (src/swpc_psv/m_wav.f90:505-532)."""
    from openswpc_b200.swpc2d import Medium2D, station_grid2d
    from oracle.oracle import Oracle2D

    p = _bd_params(custom, two_d=True)
    m = Medium2D(p)
    ist, kst = station_grid2d(p, m.kfs, m.kob)
    o = Oracle2D(p, "psv")
    n = o.nst
    oi = np.ctypeslib.as_array(C.cast(o.lib.o2d_ptr(o.o, 95), C.POINTER(C.c_int)), (n,))
    ok = np.ctypeslib.as_array(C.cast(o.lib.o2d_ptr(o.o, 96), C.POINTER(C.c_int)), (n,))
    assert len(ist) == n == len(p.stations)
    assert np.array_equal(ist, oi) and np.array_equal(kst, ok)


def test_unknown_station_mode_is_taken_as_dep_with_a_message():
    p = small3d()
    p.stations = [Station(0.3, 0.2, 2.0, "x", "bdx"), Station(0.3, 0.2, 2.0, "y", "dep")]
    m = Medium(p)
    with pytest.warns(UserWarning, match="Assume 'dep'"):
        ist, jst, kst = station_grid(p, m.kfs, m.kob)
    assert kst[0] == kst[1]


@pytest.mark.parametrize("fit", ["bd0", "bd4"])
def test_source_depth_fit_bit_exact(fit):
    """sdep_fit = 'bd<n>' moves each source to its column's boundary depth
    (m_source.f90:262-270) on both sides."""
    from openswpc_b200.swpc2d import source_grid2d
    from oracle.oracle import Oracle2D

    p = _bd_params(True)
    p.sdep_fit = fit
    p.sources = [dc_source(0.3, -0.7, 6.1, 0.0, 1.0, 1e16, 30, 60, 90),
                 Source(2.2, 1.1, 4.0, 0.2, 1.5, mo=3e15, mxx=1, myy=1, mzz=1)]
    sg = source_grid(p)
    o = Oracle3D(p)
    n = o.dims()["nsrc"]
    ks = np.ctypeslib.as_array(C.cast(o.lib.o3d_ptr(o.o, 100), C.POINTER(C.c_int)), (n,))
    assert np.array_equal(sg.ksrc, ks)
    assert sg.ksrc[0] == _lib.load().swpc_x2i(float(p.bddep[sg.jsrc[0] + 2, sg.isrc[0] + 2, int(fit[2])]),
                                              p.zbeg, p.dz)
    q = _bd_params(True, two_d=True)
    q.sdep_fit = fit
    sg2 = source_grid2d(q, "psv")
    o2 = Oracle2D(q, "psv")
    n2 = o2.nsrc
    ks2 = np.ctypeslib.as_array(C.cast(o2.lib.o2d_ptr(o2.o, 99), C.POINTER(C.c_int)), (n2,))
    assert np.array_equal(sg2.ksrc, ks2)


def test_source_depth_fit_outside_the_model_is_refused():
    """With vmodel_lhm's dummy depths (-9999) a fit to bd1 leaves FDM space,
    which source__setup asserts against (m_source.f90:276-280)."""
    p = small3d(sdep_fit="bd1")
    with pytest.raises(ValueError, match="outside the model"):
        source_grid(p)
    with pytest.raises(ValueError, match="outside the model"):
        Oracle3D(p)


def test_seawater_velocity_matches_oracle():
    """seawater__vel (src/shared/m_seawater.f90:36-49): 1.5 km/s, or Munk's
    profile (its minimum of 1.5 km/s at 1.3 km depth)."""
    lib = _lib.load()
    ol = oload()
    for z in np.linspace(0.0, 8.0, 801, dtype=np.float32):
        for munk in (0, 1):
            assert np.float32(lib.swpc_seawater_vel(float(z), munk)) == np.float32(ol.o3d_seawater_vel(float(z), munk))
    assert lib.swpc_seawater_vel(3.0, 0) == np.float32(1.5)
    assert lib.swpc_seawater_vel(1.3, 1) == np.float32(1.5)
    assert abs(lib.swpc_seawater_vel(0.0, 1) - 1.5 * (1 + 0.00737 * (np.exp(2.0) - 3.0))) < 1e-6


def _ocean(q):
    """An ocean above the layered medium: depth(1) = 1.2 km, so the cells with
    0 <= z < 1.2 km are seawater."""
    q.layers = [Layer(1.2, 2.7, 5.5, 3.2, 300, 150)] + list(q.layers[1:])
    return q


@pytest.mark.parametrize("munk", [False, True])
def test_ocean_medium_bit_exact(munk):
    """vmodel_lhm's seawater column (m_vmodel_lhm.f90:108-138) with and
    without munk_profile: every medium field and integer map of the host
    setup equals the oracle's; the ocean bottom lies below the free surface."""
    p = _ocean(small3d(munk_profile=munk))
    m = Medium(p)
    o = Oracle3D(p)
    for f in ("rho", "lam", "mu", "taup", "taus", "bx", "by", "bz", "muyz", "muxz", "muxy"):
        assert np.array_equal(bits(getattr(m, f)), bits(o.array("f" + f))), f
    for f in ("kfs", "kob", "kfs_top", "kfs_bot", "kob_top", "kob_bot"):
        assert np.array_equal(getattr(m, f), o.array(f)), f
    assert (m.kob[4:-4, 4:-4] > m.kfs[4:-4, 4:-4]).all()
    # zbeg = -1.5, dz = 0.5: cells k = 4, 5 (z = 0.25, 0.75 km) are seawater, k = 6 (1.25 km) is rock; lam is
    # the relaxed modulus of Q = 1e6, within 1e-5 of rho vp^2
    water = m.lam[5, 5, 6:8]
    assert (m.mu[5, 5, 6:8] == 0).all() and (m.rho[5, 5, 6:8] == 1).all() and m.mu[5, 5, 8] > 0
    if munk:
        assert (water > np.float32(2.25)).all() and water[0] > water[1]   # Munk's profile slows towards 1.3 km
    else:
        assert np.allclose(water, 2.25, rtol=1e-5, atol=0)


@pytest.mark.parametrize("kind", ["psv", "sh"])
def test_ocean_medium_2d_bit_exact(kind):
    from openswpc_b200.swpc2d import Medium2D
    from oracle.oracle import Oracle2D
    from tests.models import small2d

    p = _ocean(small2d(kind, munk_profile=True))
    m = Medium2D(p)
    o = Oracle2D(p, kind)
    for f in ("rho", "lam", "mu", "taup", "taus"):
        assert np.array_equal(bits(getattr(m, f)), bits(o.array("f" + f))), f
    for f in ("kfs", "kob", "kfs_top", "kfs_bot", "kob_top", "kob_bot"):
        assert np.array_equal(getattr(m, f), o.array(f)), f


def _pw_params(ps):
    """Plane-wave mode: a front at 8 km depth, 4 km long, oblique (strike 30, dip 20)."""
    return small3d(pw_mode=True, pw_ztop=8.0, pw_zlen=4.0, pw_ps=ps, pw_strike=30.0, pw_dip=20.0, pw_rake=40.0,
                   sources=[])


@pytest.mark.parametrize("ps", ["P", "S"])
def test_plane_wave_setup_bit_exact(ps):
    """pw_setup (m_source.f90:315-465): the initial V and S over the memory
    box and the PML's fcut equal the oracle's bit for bit."""
    p = _pw_params(ps)
    m = Medium(p)
    lib = _lib.load()
    f = [np.zeros(m.rho.shape, np.float32) for _ in range(9)]
    fcut = C.c_float()
    assert lib.swpc_pw_setup(C.byref(grid_struct(p)), _lib.fptr(m.rho), _lib.fptr(m.lam), _lib.fptr(m.mu),
                             p.pw_ztop, p.pw_zlen, 0 if ps == "P" else 1, p.pw_strike, p.pw_dip, p.pw_rake,
                             _lib.STF_CODES[p.stftype], *(_lib.fptr(a) for a in f), C.byref(fcut)) == 0
    o = Oracle3D(p)
    names = ["Vx", "Vy", "Vz", "Sxx", "Syy", "Szz", "Syz", "Sxz", "Sxy"]
    for a, name in zip(f, names):
        assert np.array_equal(bits(a), bits(o.array(name))), name
    assert np.abs(f[2]).max() > 0 and np.abs(f[3]).max() > 0
    sc = o.scalars()
    assert np.float32(sc["fcut"]) == np.float32(fcut.value)
    assert np.float32(sc["M0"]) == np.float32(1.0) / np.float32(1e-15)
