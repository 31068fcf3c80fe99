"""qs_sample_batched: shots of many states of uneven widths in three
launches must equal qs_sample's shot for shot, with each state's uniforms
drawn from its seed (the serving runtime's stream)."""
import numpy as np
import pytest
import torch

from qsim_b200 import engine as E

pytestmark = pytest.mark.gpu


def _states(widths, seed, scale=None):
    rng = np.random.default_rng(seed)
    offs, parts, off = [], [], 0
    for k, w in enumerate(widths):
        v = rng.normal(size=1 << w) + 1j * rng.normal(size=1 << w)
        v /= np.linalg.norm(v)
        if scale is not None:
            v *= scale[k]
        parts.append(v.astype(np.complex64))
        offs.append(off)
        off += 1 << w
    return torch.from_numpy(np.concatenate(parts)).cuda(), np.array(offs, dtype=np.int64)


@pytest.mark.parametrize("widths", [[3, 10, 15, 1, 12, 16], [7] * 40])
def test_batched_equals_per_state(widths):
    # state 2 is scaled below unit norm: its large uniforms clamp to the last index
    scale = [1.0] * len(widths)
    scale[min(2, len(widths) - 1)] = 0.6
    states, offs = _states(widths, 3, scale)
    shots = np.array([(k * 37) % 500 for k in range(len(widths))], dtype=np.int64)
    shots[1] = 0
    seeds = np.arange(len(widths), dtype=np.uint64) * np.uint64(1000003) + np.uint64(11)
    got = E.sample_batched(states, widths, offs, shots, seeds).cpu().numpy()
    assert got.shape == (int(shots.sum()),)
    k = 0
    for t, w in enumerate(widths):
        st = states[int(offs[t]): int(offs[t]) + (1 << w)]
        ref = E.sample_seeded(st, int(shots[t]), int(seeds[t])).cpu().numpy() if shots[t] else np.zeros(0)
        assert np.array_equal(got[k: k + shots[t]], ref), t
        assert got[k: k + shots[t]].max(initial=0) < (1 << w)
        k += int(shots[t])


def test_batched_edge_cases():
    states, offs = _states([4], 1)
    assert E.sample_batched(states, [4], offs, [0], [5]).numel() == 0
    assert E.sample_batched(states, [], [], [], []).numel() == 0
    with pytest.raises(ValueError):
        E.sample_batched(states, [5], offs, [3], [1])      # runs past the tensor


def test_sample_trajectories_counts():
    from qsim_b200.circuit import Circuit
    from qsim_b200.noise import run_trajectories, sample_trajectories
    qc = Circuit(3)
    qc.h(0)
    qc.cx(0, 1)
    qc.amplitude_damp(0.3, 1)
    states, _ = run_trajectories(qc, 500, seed=2, branches=False)
    counts = sample_trajectories(states, shots_per_trajectory=4, seed=9)
    assert sum(counts.values()) == 2000
    assert set(counts) <= {hex(0), hex(1), hex(2), hex(3)}
