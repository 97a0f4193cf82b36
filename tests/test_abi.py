"""The C-ABI library loads without a GPU and exports every symbol that
include/*.h declares; the ctypes structs match the header's layout."""
import ctypes as C
import glob
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for hdr in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(hdr).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"\b([A-Za-z_][\w\s\*]*?)\b(hf_\w+)\s*\(", text):
            names.add(m.group(2))
    return names


@pytest.fixture(scope="module")
def libpath():
    from hydroflux_b200 import build
    return build.build()


def test_header_declares_the_reference_surface():
    names = declared_functions()
    for must in ["hf_sim_create", "hf_sim_step", "hf_sim_run_until", "hf_sim_get_state",
                 "hf_cfl_time_step", "hf_forward_euler_step", "hf_ssprk2_step",
                 "hf_manning_friction_step", "hf_apply_rain", "hf_apply_point_sources",
                 "hf_workspace_create", "hf_last_error"]:
        assert must in names


def test_library_exports_every_declared_symbol(libpath):
    lib = C.CDLL(libpath)
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"
    out = subprocess.run(["nm", "-D", "--defined-only", libpath], capture_output=True, text=True)
    exported = {line.split()[-1] for line in out.stdout.splitlines() if " T " in line}
    assert declared_functions() <= exported


def test_prototypes_cover_header(libpath):
    from hydroflux_b200 import _lib
    assert set(_lib.PROTOTYPES) >= declared_functions()
    lib = _lib.lib()
    assert lib.hf_abi_version() == 1


def test_config_default_and_struct_layout(libpath):
    from hydroflux_b200 import _lib, abi
    cfg = abi.hf_config()
    _lib.lib().hf_config_default(C.byref(cfg))
    assert cfg.cfl == 0.4 and cfg.integrator == abi.HF_SSPRK2 and cfg.max_steps == 10_000_000
    assert cfg.max_dt == 60.0 and cfg.friction_dry_tol == 1e-6
    assert cfg.boundaries.north.kind == abi.HF_BC_WALL and cfg.boundaries.east.kind == abi.HF_BC_WALL
    assert C.sizeof(abi.hf_boundary) == 16 and C.sizeof(abi.hf_boundaries) == 64
    assert C.sizeof(abi.hf_config) == 8 + 4 + 4 + 64 + 8 + 8 + 8
    assert C.sizeof(abi.hf_mesh_desc) == 56 and C.sizeof(abi.hf_grid) == 48


def test_host_validation_without_gpu(libpath):
    """Argument checks run before any CUDA call, so they work on a CPU box."""
    from hydroflux_b200 import _lib, abi
    lib = _lib.lib()
    h = C.c_void_p()
    bad = abi.make_config(cfl=1.5)
    desc = abi.hf_mesh_desc(2, 2, 1.0, 1.0, (C.c_double * 4)(), None, 0.03)
    zeros = (C.c_double * 4)()
    rc = lib.hf_sim_create(C.byref(desc), zeros, zeros, zeros, C.byref(bad), 0, C.byref(h))
    assert rc == abi.HF_ERR_INVALID_CONFIG and b"cfl" in lib.hf_last_error()
    desc0 = abi.hf_mesh_desc(0, 2, 1.0, 1.0, (C.c_double * 4)(), None, 0.03)
    rc = lib.hf_sim_create(C.byref(desc0), zeros, zeros, zeros, C.byref(abi.make_config()), 0,
                           C.byref(h))
    assert rc == abi.HF_ERR_SHAPE_MISMATCH
    q = abi.make_boundaries((2, 1.0), (1, 0), (1, 0), (1, 0))
    desc1 = abi.hf_mesh_desc(1, 4, 1.0, 1.0, (C.c_double * 4)(), None, 0.03)
    rc = lib.hf_sim_create(C.byref(desc1), zeros, zeros, zeros,
                           C.byref(abi.make_config(boundaries=q)), 0, C.byref(h))
    assert rc == abi.HF_ERR_INVALID_CONFIG
    assert lib.hf_sim_step(None, 1.0, None) == abi.HF_ERR_INVALID_ARG
    # launch accounting: no GPU work was done, so nothing was launched
    n = C.c_uint64(7)
    assert lib.hf_kernel_launches(C.byref(n)) == abi.HF_OK and n.value == 0
    assert lib.hf_kernel_launches(None) == abi.HF_ERR_INVALID_ARG
    assert lib.hf_release_cached_memory(-1) == abi.HF_ERR_INVALID_ARG
    # Mesh2D's spacing asserts (geometry.rs:59, 93) on the device-grid entry points
    for dx, dy in ((0.0, 1.0), (1.0, -1.0), (float("nan"), 1.0)):
        g = abi.hf_grid(4, 4, dx, dy, C.c_void_p(8), C.c_void_p(8))
        rc = lib.hf_ssprk2_step_noalloc(C.byref(g), C.c_void_p(8), C.c_void_p(8), C.c_void_p(8),
                                        None, 0.1, 0, None)
        assert rc == abi.HF_ERR_INVALID_ARG and b"dx and dy" in lib.hf_last_error()


def test_manning_field_check_large(libpath):
    """Mesh2D::with_manning_field asserts n >= 0 at every cell
    (geometry.rs:103-106): the mirror's chunked check of a large field
    rejects a negative or NaN cell wherever it sits, and accepts -0.0."""
    import numpy as np
    from hydroflux_b200 import sim
    n = np.full((2048, 2560), 0.03)  # 5.2 M cells: the threaded path
    bed = np.zeros_like(n)
    sim.Mesh2D(bed, 1.0, 1.0, n)
    flat = n.reshape(-1)
    for pos in (0, 1, flat.size // 3, flat.size // 2 + 7, flat.size - 1):
        for bad in (-1e-300, float("nan"), -float("inf")):
            flat[pos] = bad
            with pytest.raises(ValueError):
                sim.Mesh2D(bed, 1.0, 1.0, n)
        flat[pos] = -0.0
        sim.Mesh2D(bed, 1.0, 1.0, n)
        flat[pos] = 0.03


def test_python_mirror_errors_without_gpu(libpath):
    import numpy as np
    from hydroflux_b200 import sim
    with pytest.raises(ValueError):
        sim.Mesh2D(np.zeros((2, 2)), 0.0, 1.0)
    with pytest.raises(ValueError):
        sim.Mesh2D(np.zeros((2, 2)), 1.0, 1.0, -0.01)
    with pytest.raises(ValueError):
        sim.Mesh2D.with_manning_field(np.zeros((3, 4)), 1.0, 1.0, np.zeros((3, 5)))
    mesh = sim.Mesh2D(np.zeros((4, 4)), 1.0, 1.0, 0.03)
    with pytest.raises(sim.InvalidConfig):
        sim.Simulation(mesh, (np.ones((4, 4)),) * 3, sim.SimulationConfig(cfl=0.0))
    with pytest.raises(sim.ShapeMismatch):
        sim.Simulation(mesh, (np.ones((3, 3)),) * 3)


def test_c99_consumer_compiles_links_and_runs(libpath):
    """The header as a foreign binding sees it: a C99 program (no C++, no CUDA
    headers) that includes it, links the library by name and calls the entry
    points that need no GPU."""
    import shutil
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("gcc not available")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = os.path.join(root, "tests", "native", "abi_consumer.c")
    out_dir = os.path.join(root, "tests", "native", "_build")
    os.makedirs(out_dir, exist_ok=True)
    exe = os.path.join(out_dir, "abi_consumer")
    libdir = os.path.dirname(libpath)
    subprocess.run([gcc, "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I",
                    os.path.join(root, "include"), src, "-L", libdir, "-lhydroflux_gpu",
                    f"-Wl,-rpath,{libdir}", "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert "abi consumer ok" in r.stdout
