"""Noisy circuits as batched stochastic trajectories.

A circuit may carry channels (``Circuit.depolarize`` / ``amplitude_damp`` /
``dephase``, the three channels of the reference's noise_sm120.cu).
``run_trajectories`` runs many independent trajectories of it in one call of
``qs_noise_trajectories``: trajectory t draws one uniform per channel, in
program order, from seed + t (splitmix64), so a trajectory's result does not
depend on how many others run with it.  Averaging over trajectories gives the
channel's density matrix; ``sample_trajectories`` draws shots from each.

    qc = add_noise(circuit, depolarizing=1e-3, amplitude_damping=2e-3)
    states, branches = run_trajectories(qc, n_traj=1024, seed=7)
    counts = sample_trajectories(states, shots_per_trajectory=4, seed=7)
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import engine as E
from .circuit import NOISE_OPS, Circuit, from_qiskit, lower
from ._lib import QsOp


def add_noise(circuit, depolarizing: float = 0.0, amplitude_damping: float = 0.0, dephasing: float = 0.0,
              qubits=None) -> Circuit:
    """A copy of `circuit` with the given channels after every gate, on each
    qubit the gate touches (in that order: depolarizing, damping, dephasing;
    a zero probability adds nothing).  qubits: restrict to these qubits."""
    circ = from_qiskit(circuit)
    keep = None if qubits is None else set(int(q) for q in qubits)
    out = Circuit(circ.num_qubits, circ.num_clbits, circ.name)
    for ins in circ.data:
        out.data.append(ins)
        if ins.name in ("barrier", "measure", "reset") or ins.name in NOISE_OPS:
            continue
        for q in ins.qubits:
            if keep is not None and q not in keep:
                continue
            if depolarizing:
                out.depolarize(depolarizing, q)
            if amplitude_damping:
                out.amplitude_damp(amplitude_damping, q)
            if dephasing:
                out.dephase(dephasing, q)
    return out


def n_channels(circuit) -> int:
    return sum(1 for ins in from_qiskit(circuit).data if ins.name in NOISE_OPS)


def run_trajectories(circuit, n_traj: int, seed: int = 0, seeds=None, device: int | None = None,
                     out: torch.Tensor | None = None, branches: bool = True):
    """(states [n_traj, 2^n] complex64 on the device, branches [n_traj,
    n_channels] uint8 or None).  Trajectory t uses seeds[t] if given, else
    seed + t.  Branch codes: depolarizing 0 = I, 1 = X, 2 = Y, 3 = Z;
    damping / dephasing 0 = no jump, 1 = jump."""
    circ = from_qiskit(circuit)
    n = circ.num_qubits
    n_traj = int(n_traj)
    dev = torch.cuda.current_device() if device is None else int(device)
    ops = np.ascontiguousarray(lower(circ))
    if seeds is None:
        seeds = np.uint64(int(seed) & (2 ** 64 - 1)) + np.arange(n_traj, dtype=np.uint64)
    seeds = np.ascontiguousarray(np.asarray(seeds, dtype=np.uint64))
    if seeds.shape != (n_traj,):
        raise ValueError("seeds must hold one seed per trajectory")
    if out is None:
        out = torch.empty((n_traj, 1 << n), dtype=torch.complex64, device=f"cuda:{dev}")
    if out.dtype != torch.complex64 or not out.is_cuda or not out.is_contiguous() or out.numel() < (n_traj << n):
        raise RuntimeError("out must be a contiguous complex64 CUDA tensor of n_traj * 2^n amplitudes")
    nn = n_channels(circ)
    br = np.zeros((n_traj, max(nn, 1)), dtype=np.uint8) if branches else None
    E._h(dev).call("qs_noise_trajectories", n, ops.ctypes.data_as(C.POINTER(QsOp)), int(len(ops)), n_traj,
                   seeds.ctypes.data_as(C.POINTER(C.c_uint64)), E._ptr(out),
                   br.ctypes.data_as(C.POINTER(C.c_uint8)) if br is not None else None)
    return out, (br[:, :nn] if br is not None else None)


def sample_trajectories(states: torch.Tensor, shots_per_trajectory: int = 1, seed: int = 0) -> dict:
    """Counts {hex(index): count} over every trajectory's shots (one batched
    sampling call; histogrammed on the device); trajectory t samples with
    the uniforms of seed + t."""
    from blackwell_backend.simulator import counts_from_samples
    T = int(states.shape[0])
    if T == 0:
        return {}
    n = int(states.shape[1]).bit_length() - 1
    seeds = np.uint64(int(seed) & (2 ** 64 - 1)) + np.arange(T, dtype=np.uint64)
    samples = E.sample_batched(states.reshape(-1), np.full(T, n), np.arange(T, dtype=np.int64) << n,
                               np.full(T, int(shots_per_trajectory)), seeds)
    return counts_from_samples(samples)
