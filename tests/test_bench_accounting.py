"""The roofline bookkeeping of bench.py: the algorithmic words per cell-step of the large step
(W(ns) = 10 + sum over the three RK stages of 50 + 20 m_s, with m_s = ceil(ns/3), ceil(ns/2), ns
acoustic substeps, as in rk3_step!, moist.jl:1589-1683) equal the per-group words times the
group's launch instances per step, so the dominant group's achieved bandwidth and the whole
step's fraction are computed from the same traffic model."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_words_per_cell_step_of_the_configs():
    assert bench.words_per_cell_step(8) == 460  # 1840 B per cell-step in Float32
    assert bench.words_per_cell_step(6) == 380  # 1520 B


@pytest.mark.parametrize("ns", range(1, 17))
def test_group_words_sum_to_the_step(ns):
    inst = bench.group_instances(ns)
    assert set(inst) == set(bench.GROUPS) == set(bench.WORDS)
    assert sum(bench.WORDS[g] * inst[g] for g in bench.GROUPS) == bench.words_per_cell_step(ns)


@pytest.mark.parametrize("ns,subs", [(1, 3), (6, 11), (8, 15), (9, 17)])
def test_substep_launches_per_step(ns, subs):
    # stages of dt/3, dt/2 and dt run max(1, ceil(ns/3)), max(1, ceil(ns/2)) and ns substeps
    assert bench.group_instances(ns)["substep"] == subs


def test_job_throughput_counts_every_replica():
    assert bench.job_throughput(262144, 4, 2e-3) == pytest.approx(4 * 262144 / 2e-3)
