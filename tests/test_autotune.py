"""Autotuner selection logic on the CPU: the GPU timing is replaced by a fake
cost table, so these check only which knobs the sweep returns."""

from __future__ import annotations

import pytest

import warpsph_b200.autotune as at
from warpsph_b200.params import SolverParams


def _run(monkeypatch, tmp_path, cost, params=None):
    monkeypatch.setattr(at, "CACHE", tmp_path / "tune.json")
    calls = []

    def fake_time(scenes, p, warm, steps):
        calls.append(p)
        return cost(p)

    monkeypatch.setattr(at, "_time", fake_time)
    params = params or SolverParams(diameter=0.02, gravity=9.81, w_table_size=1024, g_table_size=1024)
    torch = pytest.importorskip("torch")
    monkeypatch.setattr(torch.cuda, "get_device_name", lambda *a, **k: "fake")
    return at.autotune([], params, warm=1, steps=1), calls


def _shape(p):
    return (p.jacobi_block or at.DEFAULT_SOLVE[0], p.jacobi_ppt or at.DEFAULT_SOLVE[1],
            p.jacobi_unroll or at.DEFAULT_SOLVE[2])


def test_default_solve_shape_kept_when_nothing_beats_it(monkeypatch, tmp_path):
    # the build sweep (solve at the library's default shape) is fastest; every
    # other solve shape is slower, (256, 1, 2) the slowest: the default must
    # come back, not (256, 1, 2)
    def cost(p):
        if p.jacobi_block == 0:
            return 1.0
        if _shape(p) == at.DEFAULT_SOLVE:
            return 1.0
        return 3.0 if _shape(p) == (256, 1, 2) else 1.0 + 0.01 * p.jacobi_unroll

    res, _ = _run(monkeypatch, tmp_path, cost)
    assert (res["jacobi_block"], res["jacobi_ppt"], res["jacobi_unroll"]) == at.DEFAULT_SOLVE
    assert res["ms_per_step"] == 1.0


def test_fastest_solve_shape_and_build_block_chosen(monkeypatch, tmp_path):
    def cost(p):
        t = {64: 2.0, 128: 1.5, 256: 1.8}[p.block_size or 128]
        if p.jacobi_block:
            t -= 0.5 if _shape(p) == (128, 2, 8) else 0.1
        return t + (0.05 if p.plain_loads else 0.0)

    res, calls = _run(monkeypatch, tmp_path, cost)
    assert res["block_size"] == 128
    assert (res["jacobi_block"], res["jacobi_ppt"], res["jacobi_unroll"]) == (128, 2, 8)
    assert res["plain_loads"] is False
    assert len(calls) == len(at.BUILD_BLOCKS) + len(at.SOLVE_SHAPES) + 1


def test_caller_shape_is_the_baseline(monkeypatch, tmp_path):
    params = SolverParams(diameter=0.02, gravity=9.81, w_table_size=1024, g_table_size=1024,
                          jacobi_block=128, jacobi_ppt=2, jacobi_unroll=2)

    def cost(p):
        return 1.0 if _shape(p) == (128, 2, 2) else 1.2

    res, _ = _run(monkeypatch, tmp_path, cost, params)
    assert (res["jacobi_block"], res["jacobi_ppt"], res["jacobi_unroll"]) == (128, 2, 2)
