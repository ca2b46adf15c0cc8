"""CPU-only checks of the product library: exports, configuration, host-side geometry."""
import ctypes
import os
import re

import numpy as np
import pytest

from cases import CASES
from mrlbm_2d_b200.config import Config, case_large, case_mid, case_small, reference_case

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    text = open(os.path.join(ROOT, "include", "mrlbm.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|size_t)\s+(mrlbm_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol(mrlbm):
    L = mrlbm.load_library()
    syms = header_symbols()
    assert len(syms) >= 19
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(mrlbm.api.EXPORTED) | set(s for s in syms if s not in mrlbm.api.EXPORTED)


def test_config_struct_size_matches(mrlbm):
    L = mrlbm.load_library()
    L.mrlbm_config_sizeof.restype = ctypes.c_size_t
    assert L.mrlbm_config_sizeof() == ctypes.sizeof(Config)


NAMELIST = """&DomainSize
\tnx = 64
\tny = 16
\tlattice_type = 9
/
&Cylinder
\tncy = 8 ! diameter in lattice units
\tL_front = 2
\tL_back = 6
\tL_top = 1
\tL_bot = 1
/
&Numbers
\tRe = 150
/
&Parallel
\tnum_threads=4
/
&Controls
\tuo = 0.04
\trho_infty = 1.0
\tiplot = 50
\tmax_iter = 400
\tisave = 200
\tirestart = 0
\tstatsbegin =  101
\tstatsend = 300
\tiplotstats = 10
/
&LogicalControls
\tpost_process = .true.
\tx_periodic = .false.
\ty_periodic = .false.
\tchannel_with_cylinder = .true.
\tchannel_with_square = .false.
\tincomp_bc = .false.
\tincomp_bulk = .true.
\tvel_interp = .true.
\tmom_interp = .true.
\trotated_coordinate = .true.
\tstrong_mass_bc = .false.
\teq_mass_bc = .false.
\tweak_mass_bc = .true.
/
"""


def test_namelist_reader(mrlbm, tmp_path):
    p = tmp_path / "input.dat"
    p.write_text(NAMELIST)
    c = mrlbm.config_from_namelist(str(p))
    assert (c.nx, c.ny, c.ncy, c.L_front, c.L_back, c.L_top, c.L_bot) == (64, 16, 8, 2, 6, 1, 1)
    assert c.Re == 150.0 and c.uo == 0.04 and c.num_threads == 4
    assert (c.iplot, c.max_iter, c.isave, c.statsbegin, c.statsend, c.iplotstats) == (50, 400, 200, 101, 300, 10)
    assert (c.post_process, c.y_periodic, c.incomp_bulk, c.weak_mass_bc, c.strong_mass_bc) == (1, 0, 1, 1, 0)
    L = mrlbm.load_library()
    assert L.mrlbm_config_resolve_geometry(ctypes.byref(c)) == 0
    # nx = (L_front + 1 + L_back) * ncy, centre (nfront + ncy/2 + 1, nbot + ncy/2) (2d_mrlbm.f90:86-92, 946-948)
    assert (c.nx, c.ny, c.x_c, c.y_c, c.r_c) == (72, 24, 21.0, 12.0, 4.0)


@pytest.mark.parametrize("bad", ["&DomainSize\n nx = 3.5\n/\n", NAMELIST.replace("Re = 150", "Rey = 150"),
                                 NAMELIST.replace("&Controls", "&Kontrols")])
def test_namelist_errors(mrlbm, tmp_path, bad):
    p = tmp_path / "input.dat"
    p.write_text(bad)
    with pytest.raises(mrlbm.MrlbmError) as e:
        mrlbm.config_from_namelist(str(p))
    assert e.value.code == 2


def _geometry_parity(mrlbm, oracle_mod, cfg):
    s = mrlbm.Simulation(cfg, device=-1)
    o = oracle_mod.Oracle(cfg)
    b = s.boundary_nodes()
    sc = o.scalars()
    assert s.nbct == o.nbct
    assert s.info.r_cyl == sc["r_cyl"] and s.info.nu == sc["nu"] and s.info.omega == sc["omega"]
    for k in ["bou_i", "bou_j", "label_bc", "delta_uk"]:
        assert np.array_equal(b[k], o.get(k)), k
    for r in range(4):
        assert np.array_equal(b["ref_xy"][:, r], o.get(f"x_ref{r + 1}"))
        assert np.array_equal(b["ref_xy"][:, 4 + r], o.get(f"y_ref{r + 1}"))
    for r, nm in enumerate("234"):
        assert np.array_equal(b["stencil"][:, 8 * r:8 * r + 4], o.get("i_p" + nm).reshape(-1, 4))
        assert np.array_equal(b["stencil"][:, 8 * r + 4:8 * r + 8], o.get("j_p" + nm).reshape(-1, 4))
    nc = s.node_classes()
    for k in ["isfluid", "issolid", "isbound"]:
        assert np.array_equal(nc[k], o.field(k)), k
    s.close()
    return b


@pytest.mark.parametrize("name", [n for n in CASES if "no_cylinder" not in n])
def test_geometry_bit_exact_vs_oracle(mrlbm, oracle_mod, name):
    _geometry_parity(mrlbm, oracle_mod, CASES[name]())


def test_geometry_reference_default_input(mrlbm, oracle_mod):
    # the shipped input.dat: 920 x 420, centre (211, 210), r_c = 10
    b = _geometry_parity(mrlbm, oracle_mod, Config.reference_defaults())
    assert len(b["bou_i"]) == 80
    assert set(np.unique(b["label_bc"])) == {1, 2, 3, 4, 5, 7, 8, 10, 11, 12, 13, 14}


def test_geometry_benchmark_cases_host_only(mrlbm):
    # full-size benchmark geometries build on the host; label 15 appears at the two poles
    for cfg, nb in [(case_small(), 80), (case_mid(), 320), (case_large(), 1024)]:
        s = mrlbm.Simulation(cfg, device=-1)
        assert s.nbct == nb
        assert s.info.n_label15 == 2
        b = s.boundary_nodes()
        poles = {(int(i), int(j)) for i, j, l in zip(b["bou_i"], b["bou_j"], b["label_bc"]) if l == 15}
        xc, yc, r = cfg.x_c, cfg.y_c, cfg.r_c
        assert poles == {(int(xc), int(yc - r - 0.5)), (int(xc), int(yc + r + 0.5))}
        s.close()


def test_label15_rejected_in_reference_mode(mrlbm):
    cfg = case_small().replace(label15_rule=0)
    with pytest.raises(mrlbm.MrlbmError) as e:
        mrlbm.Simulation(cfg, device=-1)
    assert e.value.code == 3 and "label 15" in str(e.value)


def test_cylinder_touching_edge_rejected(mrlbm):
    cfg = case_small().replace(y_c=8.0)
    with pytest.raises(mrlbm.MrlbmError) as e:
        mrlbm.Simulation(cfg, device=-1)
    assert e.value.code == 3


def test_rotated_closure_without_moment_interp_rejected(mrlbm):
    with pytest.raises(mrlbm.MrlbmError) as e:
        mrlbm.Simulation(reference_case().replace(mom_interp=0), device=-1)
    assert e.value.code == 4


def test_host_only_handle_refuses_device_calls(mrlbm):
    s = mrlbm.Simulation(case_small(), device=-1)
    with pytest.raises(mrlbm.MrlbmError) as e:
        s.step(1)
    assert e.value.code == -3


def test_no_device_fails_loudly(mrlbm):
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(mrlbm.MrlbmError) as e:
        mrlbm.Simulation(case_small(), device=0)
    assert e.value.code in (-3, -1)


def test_header_constants_match_the_python_layer(mrlbm):
    """The #define values of include/mrlbm.h that the ctypes layer mirrors."""
    text = open(os.path.join(ROOT, "include", "mrlbm.h")).read()
    defs = {m.group(1): int(m.group(2)) for m in re.finditer(r"#define\s+(MRLBM_\w+)\s+(-?\d+)", text)}
    api = mrlbm.api
    assert defs["MRLBM_BATCH_PERSISTENT"] == api.BATCH_PERSISTENT
    assert defs["MRLBM_BATCH_GRAPH"] == api.BATCH_GRAPH
    assert defs["MRLBM_BATCH_STREAMS"] == api.BATCH_STREAMS
    assert defs["MRLBM_FP64"] == api.FP64 and defs["MRLBM_FP32"] == api.FP32


def test_batch_calls_reject_a_null_batch(mrlbm):
    """Argument checks that need no device: a NULL batch is MRLBM_EINVAL for every schedule."""
    L = mrlbm.load_library()
    text = open(os.path.join(ROOT, "include", "mrlbm.h")).read()
    einval = int(re.search(r"#define\s+MRLBM_EINVAL\s+(\d+)", text).group(1))
    for sched in (mrlbm.api.BATCH_PERSISTENT, mrlbm.api.BATCH_GRAPH, mrlbm.api.BATCH_STREAMS):
        assert L.mrlbm_batch_set_schedule(None, 7, sched, 20) == einval
    assert L.mrlbm_batch_step(None, 1, 0) == einval
