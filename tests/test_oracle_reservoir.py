"""Reservoir algebra of ReSTIR DI: the oracle restatement (oracle/reservoir.py)
against the reference's own DirectLightReservoir, replayed from
tests/golden/reservoir.json (made by tests/golden/make_reservoir_golden.py),
and in the device's float32 arithmetic."""
import json

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import reservoir as rv


@pytest.fixture(scope="module")
def cases():
    return json.loads((GOLDEN / "reservoir.json").read_text())


def _stream(cands, dtype=np.float64):
    res = rv.Reservoir()
    selected = []
    for c in cands:
        cand = rv.Candidate(c["light"], c["u"], c["v"], c["target"])
        selected.append(rv.stream(res, cand, c["weight"], c["random"], represented=c["represented"], dtype=dtype))
    return res, selected


def _summary(res, dtype=np.float64):
    return {"light": -1 if res.sample is None else res.sample.light,
            "target": 0.0 if res.sample is None else float(res.sample.target),
            "weight_sum": float(res.weight_sum), "count": res.count,
            "normalization": rv.contribution_weight(res, dtype=dtype)}


def test_streams_select_the_reference_samples(cases):
    for case in cases["streams"]:
        res, selected = _stream(case["candidates"])
        assert selected == case["selected"]
        assert _summary(res) == case["final"]


def test_reuse_chains_equal_the_reference_merges(cases):
    for case in cases["reuses"]:
        dest, selected = _stream(case["destination"])
        assert selected == case["destination_selected"]
        sources = []
        for src in case["sources"]:
            res, _ = _stream(src["candidates"])
            assert _summary(res) == src["final"]
            sources.append(res)
        for m in case["merges"]:
            assert rv.reuse(dest, sources[m["source"]], m["target_here"], m["random"]) == m["reused"]
        assert _summary(dest) == case["final"]


def test_device_float32_arithmetic_keeps_the_selections(cases):
    """The kernels sum and compare in float32: the same samples win except
    where u * weight_sum and the weight tie to float32 precision."""
    checked = 0
    for case in cases["streams"]:
        res64, sel64 = _stream(case["candidates"])
        res32, sel32 = _stream(case["candidates"], dtype=np.float32)
        ws = 0.0
        robust = True
        for c, a, b in zip(case["candidates"], sel64, sel32):
            ws += c["weight"]
            if c["weight"] > 0.0 and abs(c["random"] * ws - c["weight"]) <= 1e-5 * ws:
                robust = False
            if robust:
                assert a == b
        if robust:
            checked += 1
            assert _summary(res32)["light"] == case["final"]["light"]
            np.testing.assert_allclose(float(res32.weight_sum), case["final"]["weight_sum"], rtol=1e-5)
            np.testing.assert_allclose(rv.contribution_weight(res32, dtype=np.float32),
                                       case["final"]["normalization"], rtol=1e-5)
    assert checked == len(cases["streams"])


def test_weighted_stream_tracks_sum_count_and_weight():
    res = rv.Reservoir()
    first = rv.Candidate(7, 0.25, 0.5, 1.5)
    second = rv.Candidate(9, 0.125, 0.25, 3.0)
    assert rv.stream(res, first, 2.0, 0.9)            # nothing held yet: any positive weight wins
    assert rv.stream(res, second, 6.0, 0.2)           # 0.2 * 8 = 1.6 < 6
    assert res.sample == second and res.weight_sum == 8.0 and res.count == 2
    assert rv.contribution_weight(res) == 8.0 / (2 * 3.0)
    third = rv.Candidate(11, 0.5, 0.5, 1.0)
    assert not rv.stream(res, third, 1.0, 0.5)        # 0.5 * 9 = 4.5 >= 1
    assert res.sample == second and res.count == 3


def test_zero_weight_candidate_is_counted_but_never_held():
    res = rv.Reservoir()
    assert not rv.stream(res, rv.Candidate(3, 0.1, 0.2, 0.0), 0.0, 0.0)
    assert res.sample is None and res.count == 1 and res.weight_sum == 0.0
    assert rv.contribution_weight(res) == 0.0


def test_reuse_reweights_by_the_target_at_this_surface():
    source = rv.Reservoir(rv.Candidate(4, 0.3, 0.3, 2.0), 10.0, 5)
    dest = rv.Reservoir()
    assert rv.reuse(dest, source, 3.0, 0.5)
    # weight = 3 * 10 / 2 = 15, representing the source's 5 samples
    assert dest.weight_sum == 15.0 and dest.count == 5
    assert dest.sample.light == 4 and dest.sample.target == 3.0
    assert rv.contribution_weight(dest) == 15.0 / (5 * 3.0)


def test_reuse_of_an_empty_source_changes_nothing():
    dest = rv.Reservoir(rv.Candidate(1, 0.0, 0.0, 1.0), 2.0, 3)
    assert not rv.reuse(dest, rv.Reservoir(), 5.0, 0.1)
    assert dest.weight_sum == 2.0 and dest.count == 3


def test_history_clamp_scales_the_weight_sum():
    prev = rv.Reservoir(rv.Candidate(2, 0.5, 0.25, 1.0), 50.0, 100)
    capped = rv.cap_history(prev, 20)
    assert capped.count == 20 and capped.weight_sum == pytest.approx(10.0)
    assert rv.cap_history(prev, 1000).count == 100
    # W is unchanged by the clamp
    assert rv.contribution_weight(capped) == pytest.approx(rv.contribution_weight(prev))


@pytest.mark.parametrize("call", [
    lambda: rv.stream(rv.Reservoir(), rv.Candidate(0, 0, 0, 1.0), -1.0, 0.5),
    lambda: rv.stream(rv.Reservoir(), rv.Candidate(0, 0, 0, 1.0), float("nan"), 0.5),
    lambda: rv.stream(rv.Reservoir(), rv.Candidate(0, 0, 0, 1.0), 1.0, 1.0),
    lambda: rv.stream(rv.Reservoir(), rv.Candidate(0, 0, 0, 1.0), 1.0, 0.5, represented=0),
    lambda: rv.Candidate(-1, 0, 0, 1.0),
    lambda: rv.Candidate(0, 0, 0, float("inf")),
    lambda: rv.reuse(rv.Reservoir(), rv.Reservoir(rv.Candidate(0, 0, 0, 1.0), 1.0, 1), -2.0, 0.5),
])
def test_invalid_inputs_raise_like_the_reference(call):
    with pytest.raises(ValueError):
        call()
