"""Bookkeeping of bench.py that needs no GPU: the DRAM traffic figures it
reports come from committed ncu summaries of the build it names and lie
where the kernel's design puts them, and the algorithmic bytes per cell
follow B_alg = 2 (Q s_f + 7 s_g + 4)."""
import importlib.util
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_traffic_figures_come_from_their_profiles():
    bench = load_bench()
    assert bench.NCU_BYTES_PER_CELL
    for (q, storage), (per_cell, path, build) in bench.NCU_BYTES_PER_CELL.items():
        text = open(os.path.join(ROOT, path)).read()
        # the summary names the kernel instantiation, the build and the per-cell figure
        assert f"bulk_kernel<{q}," in text, path
        assert f"Build {build}" in text, (path, build)
        assert re.search(r"\*\*%.1f B\*\*" % per_cell, text), (path, per_cell)
        # the figure lies between the population bytes (phi is rebuilt from g,
        # not stored; lines still dirty in L2 at the end are counted later)
        # and B_alg, which counts a phi read and write as well
        s_f, s_g = bench.element_sizes(bench.STORAGE_NAMES[storage])
        alg = bench.b_alg(q, s_f, s_g)
        populations = alg - 8
        assert 0.98 * populations <= per_cell <= 1.01 * alg, (per_cell, populations, alg)


def test_algorithmic_bytes_per_cell():
    bench = load_bench()
    assert bench.b_alg(27, 4, 4) == 280
    assert bench.b_alg(19, 4, 4) == 216
    assert bench.b_alg(27, 2, 2) == 144
    assert bench.b_alg(19, 2, 2) == 112
