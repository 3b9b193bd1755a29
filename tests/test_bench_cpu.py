"""The algorithmic byte counts behind every T_eff figure of bench.py (no GPU
needed): the minimum field elements one PT iteration must move, counted field by
field at the exact staggered interior sizes."""
import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def staggered_sizes(n):
    nx, ny, nz = n
    return {
        "P": nx * ny * nz, "txx": nx * ny * nz, "tyy": nx * ny * nz, "tzz": nx * ny * nz,
        "txy": (nx + 1) * (ny + 1) * nz, "txz": (nx + 1) * ny * (nz + 1), "tyz": nx * (ny + 1) * (nz + 1),
        "Vx": (nx + 1) * ny * nz, "Vy": nx * (ny + 1) * nz, "Vz": nx * ny * (nz + 1),
        "eta": nx * ny * nz,
    }


def test_a_eff_counts_22_passes_at_staggered_sizes():
    b = load_bench()
    for n in ((511, 511, 511), (255, 127, 63), (3, 4, 5)):
        s = staggered_sizes(n)
        state = sum(v for k, v in s.items() if k != "eta")
        # P, τ and V read and written; η read; η_next written
        assert b.a_eff_elements(n) == 2 * state + 2 * s["eta"]
    # 511^3 in FP64: the 23.52 GB per iteration the headline T_eff divides
    assert b.a_eff_elements((511, 511, 511)) * 8 == 23_521_804_208


def test_immersed_boundary_a_eff_adds_fourteen_mask_reads():
    b = load_bench()
    n = (383, 383, 383)
    nx, ny, nz = n
    masks = (nx * ny * nz + (nx + 1) * ny * nz + nx * (ny + 1) * nz + nx * ny * (nz + 1)
             + (nx + 1) * (ny + 1) * nz + (nx + 1) * ny * (nz + 1) + nx * (ny + 1) * (nz + 1))
    assert b.ib_a_eff_elements(n) == b.a_eff_elements(n) + 2 * masks
