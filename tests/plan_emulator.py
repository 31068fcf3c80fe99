"""Host emulation (FP64) of the device program the planner emits.

The library exports the program it would upload (`qs_plan_program`): passes
back to back, each a header, register blocks, ops and a coefficient pool.
This module decodes it and applies every op of every block of every pass to a
full complex128 state, with the op semantics of the tile-pass kernel
(qiskit-blackwell_b200/csrc/qs_pass.cu).  Run in FP64 with the FP32
coefficients, it checks the planner's algebra (fusion, rotation
decomposition, scaled rotations, diagonal merging, pass split) to ~1e-7
without a GPU; the GPU tests then check the kernels against the same oracle.

Blocks of a pass act on disjoint amplitude groups of each tile and every op
only mixes amplitudes inside one group, so applying each op to the whole
state in program order is the same computation as the kernel's tile loop.
"""
import ctypes as C

import numpy as np

from qsim_b200 import _lib

PASS_DT = np.dtype([("T", "<i4"), ("R", "<i4"), ("nblocks", "<i4"), ("n_qubits", "<i4"), ("S", "<i4", 16),
                    ("block_off", "<u4"), ("op_off", "<u4"), ("coef_off", "<u4"), ("bytes", "<u4"),
                    ("ncoef", "<u4"), ("has2", "<u4"), ("pad", "<u4", 2)])
BLOCK_DT = np.dtype([("pos", "i1", 8), ("op_begin", "<i4"), ("op_end", "<i4")])
# DevOp is declared __align__(16): 24 bytes of fields padded to 32
OP_DT = np.dtype({"names": ["kind", "t0", "t1", "rc", "d0", "d1", "ncoef", "pad0", "coef", "pad1", "gc"],
                  "formats": ["u1", "u1", "u1", "u1", "u1", "u1", "u1", "u1", "<u4", "<u4", "<u8"],
                  "offsets": [0, 1, 2, 3, 4, 5, 6, 7, 8, 12, 16], "itemsize": 32})
assert PASS_DT.itemsize == 112 and BLOCK_DT.itemsize == 16

DK_U1, DK_U2, DK_X, DK_SWAP, DK_Y = 1, 2, 3, 4, 5
DK_RY, DK_DTAB, DK_KRY, DK_KU1, DK_SCALE, DK_XRY, DK_CU2, DK_NOISE = 10, 11, 12, 13, 14, 15, 16, 17


def program(n, ops, tile_bits=0, block_bits=0, specialised=False) -> bytes:
    L = _lib.load()
    ops = np.ascontiguousarray(ops)
    p = ops.ctypes.data_as(C.POINTER(_lib.QsOp))
    need = C.c_size_t(0)
    sp = int(bool(specialised))
    _lib.check(L.qs_plan_program(n, p, len(ops), tile_bits, block_bits, sp, None, 0, C.byref(need)))
    buf = (C.c_char * max(1, need.value))()
    _lib.check(L.qs_plan_program(n, p, len(ops), tile_bits, block_bits, sp, buf, need.value, C.byref(need)))
    return bytes(buf)[: need.value]


def decode(blob: bytes):
    """-> list of passes: (header, blocks, ops, coefficient pool as raw float32 pairs)."""
    out, off = [], 0
    while off < len(blob):
        hdr = np.frombuffer(blob, PASS_DT, 1, off)[0]
        nb = int(hdr["nblocks"])
        blocks = np.frombuffer(blob, BLOCK_DT, nb, off + int(hdr["block_off"]))
        nops = int(blocks["op_end"].max()) if nb else 0
        dops = np.frombuffer(blob, OP_DT, nops, off + int(hdr["op_off"]))
        raw = np.frombuffer(blob, "<f4", 2 * int(hdr["ncoef"]), off + int(hdr["coef_off"]))
        out.append((hdr, blocks, dops, raw))
        off += int(hdr["bytes"])
    return out


def _bits(raw, k):
    """Coefficient slot k read as raw 32-bit words (masks stored in the pool)."""
    w = raw[2 * k: 2 * k + 2].view("<u4")
    return int(w[0]), int(w[1])


def noise_program(n, ops, block_bits=0) -> bytes:
    """The whole-state program `qs_noise_trajectories` runs (n <= 14)."""
    L = _lib.load()
    ops = np.ascontiguousarray(ops)
    p = ops.ctypes.data_as(C.POINTER(_lib.QsOp))
    need = C.c_size_t(0)
    _lib.check(L.qs_noise_program(n, p, len(ops), block_bits, None, 0, C.byref(need)))
    buf = (C.c_char * max(1, need.value))()
    _lib.check(L.qs_noise_program(n, p, len(ops), block_bits, buf, need.value, C.byref(need)))
    return bytes(buf)[: need.value]


def run(n, blob: bytes, psi: np.ndarray, seed=None, branches=None) -> np.ndarray:
    """Apply the program to psi.  Noise blocks draw channel k's uniform as
    value k of `seed`'s splitmix64 stream and append (k, branch) to
    `branches` when it is a list."""
    psi = np.array(psi, dtype=np.complex128)
    idx = np.arange(1 << n, dtype=np.uint64)
    for hdr, blocks, dops, raw in decode(blob):
        S = [int(x) for x in hdr["S"][: int(hdr["T"])]]
        R = int(hdr["R"])
        cf = raw[0::2].astype(np.float64) + 1j * raw[1::2].astype(np.float64)
        for b in blocks:
            if int(b["pos"][6]):
                assert seed is not None, "a noise program needs a seed"
                psi = _noise_block(psi, idx, S, b, dops, int(seed), branches)
                continue
            regq = [S[int(p)] for p in b["pos"][:R]]
            rmask = 0
            for q in regq:
                rmask |= 1 << q
            gidx = idx & np.uint64(~rmask & ((1 << 64) - 1))
            need_g = int(b["pos"][7]) != 0
            if not need_g:
                gidx = np.zeros_like(idx)
            # register index j of each amplitude
            jreg = np.zeros(1 << n, dtype=np.int64)
            for k, q in enumerate(regq):
                jreg |= ((idx >> np.uint64(q)) & np.uint64(1)).astype(np.int64) << k
            for o in dops[int(b["op_begin"]): int(b["op_end"])]:
                psi = _apply(psi, o, cf, raw, regq, R, idx, gidx, jreg)
    return psi


def _uniform_at(seed, k):
    """Value k of splitmix64 from seed (Steele, Lea and Flood, 2014), top 53
    bits scaled to [0, 1)."""
    m = (1 << 64) - 1
    z = (seed + (k + 1) * 0x9E3779B97F4A7C15) & m
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & m
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & m
    z ^= z >> 31
    return (z >> 11) * 2.0 ** -53


def _depol_branch(p, u):
    if u < 1.0 - p:
        return 0
    r, third = u - (1.0 - p), p / 3.0
    return 1 if r < third else (2 if r < 2.0 * third else 3)


def _noise_block(psi, idx, S, b, dops, seed, branches):
    """A noise block as the kernel runs it: the bin histogram of |a|^2 over
    the block's qubits Q, every channel's branch decided in order from the
    running histogram, and the composed map a'(i) = C[bin(i)] a(i ^ M)
    applied once with C rounded to FP32."""
    nq = int(b["pos"][5])
    pos = [int(x) for x in b["pos"][:nq]]
    Q = [S[p] for p in pos]
    NB = 1 << nq
    binv = np.zeros(idx.shape, dtype=np.int64)
    for j, q in enumerate(Q):
        binv |= ((idx >> np.uint64(q)) & np.uint64(1)).astype(np.int64) << j
    ops = dops[int(b["op_begin"]): int(b["op_end"])]
    H = np.bincount(binv, weights=np.abs(psi) ** 2, minlength=NB)
    C = np.ones(NB, dtype=np.complex128)
    bins = np.arange(NB)
    Mb, ident = 0, True
    for o in ops:
        assert int(o["kind"]) == DK_NOISE
        j = pos.index(int(o["t0"]))
        bit = 1 << j
        st = (bins & bit) != 0
        g = float(np.array([int(o["gc"])], dtype=np.uint64).view(np.float64)[0])
        k = int(o["coef"])
        u = _uniform_at(seed, k)
        m, c = 0, np.ones(NB, dtype=np.complex128)
        if int(o["d0"]) == 20:
            br = _depol_branch(g, u)
            if branches is not None:
                branches.append((k, br))
            if br == 0:
                continue
            if br == 1:
                m = bit
            elif br == 2:
                m, c = bit, np.where(st, 1j, -1j)
            else:
                c = np.where(st, -1.0, 1.0).astype(np.complex128)
        else:
            S0, S1 = float(H[~st].sum()), float(H[st].sum())
            p1 = g * S1 / (S0 + S1)
            keep = S0 + (1.0 - g) * S1
            jump = S1 > 0.0 and (u < p1 or not keep > 0.0)
            if branches is not None:
                branches.append((k, int(jump)))
            if not jump:
                r = 1.0 / np.sqrt(keep)
                c = np.where(st, np.sqrt(1.0 - g) * r, r).astype(np.complex128)
            elif int(o["d0"]) == 21:
                m, c = bit, np.where(st, 0.0, 1.0 / np.sqrt(S1)).astype(np.complex128)
            else:
                c = np.where(st, 1.0 / np.sqrt(S1), 0.0).astype(np.complex128)
        ident = False
        C = c * C[bins ^ m]
        H = np.abs(c) ** 2 * H[bins ^ m]
        Mb ^= m
    if ident:
        return psi
    C = C.astype(np.complex64).astype(np.complex128)
    flip = 0
    for j, q in enumerate(Q):
        if (Mb >> j) & 1:
            flip |= 1 << q
    return C[binv] * psi[(idx ^ np.uint64(flip)).astype(np.int64)]


def _pairs(idx, q):
    m = np.uint64(1 << q)
    lo = idx[(idx & m) == 0]
    return lo, lo | m


def _pred(o, regq, idx, gidx, base):
    """Controls of op o evaluated at the amplitudes `base` (target bits 0)."""
    ok = np.ones(base.shape, dtype=bool)
    rc = int(o["rc"])
    for k, q in enumerate(regq):
        if (rc >> k) & 1:
            ok &= ((base >> np.uint64(q)) & np.uint64(1)) == 1
    gc = np.uint64(int(o["gc"]))
    if int(o["gc"]):
        ok &= (gidx[base.astype(np.int64)] & gc) == gc
    return ok


def _apply(psi, o, cf, raw, regq, R, idx, gidx, jreg):
    kind, c0 = int(o["kind"]), int(o["coef"])
    if kind in (DK_U1, DK_RY, DK_X, DK_Y):
        q = regq[int(o["t0"])]
        i0, i1 = _pairs(idx, q)
        p = _pred(o, regq, idx, gidx, i0)
        i0, i1 = i0[p].astype(np.int64), i1[p].astype(np.int64)
        a0, a1 = psi[i0].copy(), psi[i1].copy()
        if kind == DK_U1:
            g = cf[c0: c0 + 4]
            psi[i0], psi[i1] = g[0] * a0 + g[1] * a1, g[2] * a0 + g[3] * a1
        elif kind == DK_RY:
            co, si = raw[2 * c0], raw[2 * c0 + 1]
            psi[i0], psi[i1] = co * a0 - si * a1, si * a0 + co * a1
        elif kind == DK_X:
            psi[i0], psi[i1] = a1, a0
        else:
            psi[i0], psi[i1] = -1j * a1, 1j * a0
        return psi
    if kind in (DK_KRY, DK_KU1):
        mask = int(o["t0"])
        for K in range(R):
            if not (mask >> K) & 1:
                continue
            i0, i1 = _pairs(idx, regq[K])
            i0, i1 = i0.astype(np.int64), i1.astype(np.int64)
            a0, a1 = psi[i0].copy(), psi[i1].copy()
            if kind == DK_KRY:
                t, form = float(raw[2 * (c0 + K)]), float(raw[2 * (c0 + K) + 1])
                if form == 0.0:
                    psi[i0], psi[i1] = a0 - t * a1, a1 + t * a0
                else:
                    psi[i0], psi[i1] = t * a0 - a1, a0 + t * a1
            else:
                g = cf[c0 + 4 * K: c0 + 4 * K + 4]
                psi[i0], psi[i1] = g[0] * a0 + g[1] * a1, g[2] * a0 + g[3] * a1
        return psi
    if kind == DK_SCALE:
        return psi * float(raw[2 * c0])
    if kind == DK_XRY:
        qa, qb = regq[int(o["t0"])], regq[int(o["t1"])]
        ma, mb = np.uint64(1 << qa), np.uint64(1 << qb)
        for par in (0, 1):   # 0: (|00>, |11>), 1: (|qa=0 qb=1>, |qa=1 qb=0>)
            x = idx[((idx & ma) == 0) & (((idx & mb) != 0) == bool(par))]
            y = x ^ (ma | mb)
            x, y = x.astype(np.int64), y.astype(np.int64)
            t, form = float(raw[2 * (c0 + par)]), float(raw[2 * (c0 + par) + 1])
            a0, a1 = psi[x].copy(), psi[y].copy()
            if form == 0.0:
                psi[x], psi[y] = a0 - t * a1, a1 + t * a0
            else:
                psi[x], psi[y] = t * a0 - a1, a0 + t * a1
        return psi
    if kind in (DK_U2, DK_CU2, DK_SWAP):
        qa, qb = regq[int(o["t0"])], regq[int(o["t1"])]
        ma, mb = np.uint64(1 << qa), np.uint64(1 << qb)
        base = idx[((idx & ma) == 0) & ((idx & mb) == 0)]
        p = _pred(o, regq, idx, gidx, base)
        base = base[p]
        ii = [base.astype(np.int64), (base | ma).astype(np.int64), (base | mb).astype(np.int64),
              (base | ma | mb).astype(np.int64)]
        a = [psi[i].copy() for i in ii]
        if kind == DK_SWAP:
            psi[ii[1]], psi[ii[2]] = a[2], a[1]
        else:
            g = cf[c0: c0 + 16].reshape(4, 4)
            for r in range(4):
                psi[ii[r]] = g[r, 0] * a[0] + g[r, 1] * a[1] + g[r, 2] * a[2] + g[r, 3] * a[3]
        return psi
    if kind == DK_DTAB:
        J = 1 << R
        k = c0
        table = int(o["rc"]) & 1
        t = np.ones(psi.shape, dtype=np.complex128)
        if table:
            t = cf[k: k + J][jreg]
            k += J
        for _ in range(int(o["t0"])):
            lo, hi = _bits(raw, k)
            gm = np.uint64(lo | (hi << 32))
            t = np.where((gidx & gm) == gm, t * cf[k + 1], t)
            k += 2
        m = np.zeros(psi.shape, dtype=np.uint64)
        for _ in range(int(o["t1"])):
            rlo, rhi = _bits(raw, k)
            rm = rlo | (rhi << 32)
            lo, hi = _bits(raw, k + 1)
            gm = np.uint64(lo | (hi << 32))
            m = np.where((gidx & gm) == gm, m ^ np.uint64(rm), m)
            k += 2
        sign = np.where((m >> jreg.astype(np.uint64)) & np.uint64(1), -1.0, 1.0)
        psi = psi * t * sign
        for _ in range(int(o["d0"])):
            rlo, rhi = _bits(raw, k)
            rm = rlo | (rhi << 32)
            lo, hi = _bits(raw, k + 1)
            gm = np.uint64(lo | (hi << 32))
            w = cf[k + 2]
            hit = ((gidx & gm) == gm) & (((np.uint64(rm) >> jreg.astype(np.uint64)) & np.uint64(1)) == 1)
            psi = np.where(hit, psi * w, psi)
            k += 3
        return psi
    raise ValueError(f"unknown device op kind {kind}")
