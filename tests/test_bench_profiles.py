"""The bench line's roofline figures come from the committed ncu summaries:
every stage kernel the bench can name has its per-cell DRAM traffic and its
warp instructions per cell-update there, and each simulation stage kind maps
to one of those names (no GPU needed)."""
import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_every_stage_kernel_has_profiled_figures():
    bench = load_bench()
    from hydroflux_b200.sim import Simulation
    kinds = set(Simulation.STAGE_KERNELS) - {"auto"}
    assert kinds == set(bench.KERNEL_NAMES)
    for kind, name in bench.KERNEL_NAMES.items():
        traffic = bench.profiled_traffic(name)
        per_cell = bench.profiled_figure(name, "warp_instructions_per_cell_update")
        assert traffic is not None and 40.0 < traffic < 80.0, (kind, traffic)
        assert per_cell is not None and 100.0 < per_cell < 300.0, (kind, per_cell)


def test_profile_summaries_name_their_commands():
    """Each committed summary names the command that made it and holds no
    raw report."""
    prof = os.path.join(ROOT, "profiles")
    for f in sorted(os.listdir(prof)):
        path = os.path.join(prof, f)
        assert f.endswith((".md", ".txt")), f
        assert os.path.getsize(path) < 20000, f
        if f.endswith(".md"):
            text = open(path).read()
            assert "ncu " in text and "--clock-control none" in text, f
