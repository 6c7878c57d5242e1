"""Host logic of the block-size and member-tile autotuner (cmfb200.autotune)
on a stand-in model with fixed per-candidate times, no GPU: the candidate
grid (member tiles that divide the member count, one tile for one member),
the pick, the state restore after every candidate, the restore after a
failing or invalid candidate, and the JSON cache."""
import json

import pytest
import torch

from cmfb200 import autotune as AT


class StandInModel:
    """The attributes and calls tune_block_size uses, on the CPU."""

    def __init__(self, members: int, block: int = 256):
        self.num_members = members
        self.block_size = block
        self.member_tile = 1
        self.device = torch.device("cpu")
        self.state = {"river_storage": torch.arange(6, dtype=torch.float64)}
        self.timed = []

    def state_tensors(self):
        return self.state

    def _rebuild_plan(self, block_size: int) -> None:   # keeps the member tile
        self.block_size = int(block_size)

    def set_member_tile(self, width: int) -> None:
        if self.num_members % width:
            raise ValueError(width)
        self.member_tile = int(width)


def _fake_timer(table, fail_block=None):
    def timer(model, sub_steps, repeats):
        if model.block_size == fail_block:
            raise RuntimeError("launch failed")
        model.timed.append((model.block_size, model.member_tile))
        model.state["river_storage"] += 1.0             # the trial sub-steps move the state
        return table(model.block_size, model.member_tile)
    return timer


@pytest.fixture(autouse=True)
def _no_gpu_key(monkeypatch):
    monkeypatch.setattr(AT, "_cache_key", lambda m: f"stand-in|M={m.num_members}")


def test_member_tiles_dividing_the_member_count(monkeypatch):
    monkeypatch.setattr(AT, "_time_candidate",
                        _fake_timer(lambda b, w: abs(b - 128) + 10.0 / w if w != 4 else 99.0))
    m = StandInModel(members=4)
    before = m.state["river_storage"].clone()
    res = AT.tune_block_size(m, candidates=(64, 128, 256))
    assert sorted(set(m.timed)) == sorted((b, w) for b in (64, 128, 256) for w in (1, 2, 4))
    assert (res["block_size"], res["member_tile"]) == (128, 2)
    assert (m.block_size, m.member_tile) == (128, 2)
    assert set(res["ms_per_sub_step"]) == {f"{b}/{w}" for b in (64, 128, 256) for w in (1, 2, 4)}
    assert torch.equal(m.state["river_storage"], before)
    assert not res["cached"]


def test_one_member_searches_block_size_only(monkeypatch):
    monkeypatch.setattr(AT, "_time_candidate", _fake_timer(lambda b, w: float(b)))
    m = StandInModel(members=1)
    res = AT.tune_block_size(m, candidates=(128, 64, 256), tile_candidates=(1, 2, 4))
    assert m.timed == [(128, 1), (64, 1), (256, 1)]
    assert res["block_size"] == 64 and res["member_tile"] == 1
    assert set(res["ms_per_sub_step"]) == {128, 64, 256}


@pytest.mark.parametrize("bad", ["fail", "invalid"])
def test_failure_restores_plan_and_state(bad, monkeypatch):
    monkeypatch.setattr(AT, "_time_candidate",
                        _fake_timer(lambda b, w: 1.0, fail_block=192 if bad == "fail" else None))
    m = StandInModel(members=2, block=256)
    m.member_tile = 2
    before = m.state["river_storage"].clone()
    cands = (64, 192) if bad == "fail" else (64, 48)
    with pytest.raises(RuntimeError if bad == "fail" else ValueError):
        AT.tune_block_size(m, candidates=cands)
    assert (m.block_size, m.member_tile) == (256, 2)
    assert torch.equal(m.state["river_storage"], before)


def test_cache_round_trip(monkeypatch, tmp_path):
    monkeypatch.setattr(AT, "_time_candidate", _fake_timer(lambda b, w: b / w))
    cache = tmp_path / "tune.json"
    m = StandInModel(members=8)
    res = AT.tune_block_size(m, candidates=(64, 256), tile_candidates=(1, 8), cache_path=str(cache))
    assert (res["block_size"], res["member_tile"]) == (64, 8)
    stored = json.loads(cache.read_text())["stand-in|M=8"]
    assert stored["block_size"] == 64 and stored["member_tile"] == 8
    fresh = StandInModel(members=8)
    again = AT.tune_block_size(fresh, candidates=(64, 256), cache_path=str(cache))
    assert again["cached"] and fresh.timed == []
    assert (fresh.block_size, fresh.member_tile) == (64, 8)
