// qs_noise.cu — stochastic noise channels.
//
// Two entry levels:
//  * one channel on one state, with the reference's semantics and branch
//    encoding (bwk/csrc/noise_sm120.cu:238-373): depolarizing is chosen on
//    the host from the caller's uniform and applied as an exact Pauli;
//    amplitude damping and dephasing need P(q=1) of the current state, which
//    is reduced in FP64 on the device and compared with the uniform there, so
//    nothing waits for the host unless the caller asks for the branch;
//  * batched trajectories of one noisy circuit.  Trajectory t's uniform for
//    channel k is number k of the splitmix64 stream of its seed, computed
//    where it is used, so a trajectory's result does not depend on the
//    batch it runs in:
//      - up to 14 qubits a trajectory's state is one shared-memory tile, so
//        every channel is a "noise block" inside the tile-pass program
//        (qs_pass.cu: the depolarizing Pauli, or a CTA-wide FP64 reduction,
//        the branch and the Kraus operator).  One program serves all
//        trajectories; a whole noisy circuit runs start to finish in one CTA
//        per trajectory, all trajectories in one launch per program level;
//      - wider states run the unitary segments between state-dependent
//        channels as batch launches and each such channel as two launches
//        over all trajectories (per-block FP64 partial sums, then branch +
//        Kraus operator).  There depolarizing outcomes are drawn on the host
//        and become Paulis that the FP64 planner fuses with the gates
//        (trajectories with the same outcomes share a program).
#include "qs_api.h"
#include "qs_common.cuh"
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>

using namespace qs;

namespace {

constexpr int kThreads = 256;

// CTA size of the whole-state trajectory launches: 128 (measured on B200
// against 64 and 256 on a 12-qubit, 840-channel circuit); QSIM_NOISE_THREADS
// overrides (a multiple of 32; 0 = the tile-pass default).
int noise_threads() {
  const char* e = std::getenv("QSIM_NOISE_THREADS");
  return e ? std::atoi(e) : 128;
}

bool is_noise(int kind) {
  return kind == QS_OP_DEPOLARIZE || kind == QS_OP_AMP_DAMP || kind == QS_OP_DEPHASE;
}

// Exact Paulis on one state: 1 = X, 2 = Y, 3 = Z.
__global__ void k_pauli(float2* __restrict__ s, int q, int kind, uint64_t npairs) {
  for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < npairs;
       c += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i0 = insert_zero(c, q), i1 = i0 | (1ull << q);
    const float2 a1 = s[i1];
    if (kind == 3) {
      s[i1] = make_float2(-a1.x, -a1.y);
      continue;
    }
    const float2 a0 = s[i0];
    if (kind == 1) {
      s[i0] = a1;
      s[i1] = a0;
    } else {  // Y = [[0, -i], [i, 0]]
      s[i0] = make_float2(a1.y, -a1.x);
      s[i1] = make_float2(-a0.y, a0.x);
    }
  }
}

// Blocks per state for the two-launch channel: a power of two, at most
// 2^(n-1) (so every block owns at least one amplitude pair) and 1024, with
// at least 8 amplitudes per thread.
int blocks_per_state(int n) {
  int b = 1;
  while (b < 1024 && ((uint64_t)b << 1) <= (1ull << (n - 1)) &&
         ((1ull << n) / ((uint64_t)b << 1)) >= (uint64_t)kThreads * 8)
    b <<= 1;
  return b;
}

// partials[t * bpt + b] = (S0, S1): sums of |a|^2 over the q = 0 / q = 1
// amplitudes of block b's chunk of state t (fixed order: per thread, warps
// in index order).
__global__ void __launch_bounds__(kThreads) k_noise_sums(const float2* __restrict__ states, int n, int q, int bpt,
                                                         double2* __restrict__ partials, int t0) {
  const int t = t0 + blockIdx.y, b = blockIdx.x;
  const uint64_t N = 1ull << n, chunk = N / (uint64_t)bpt;
  const uint64_t base = (uint64_t)b * chunk;
  const float2* s = states + (uint64_t)t * N + base;
  double s0 = 0.0, s1 = 0.0;
  for (uint64_t i = threadIdx.x; i < chunk; i += blockDim.x) {
    const float2 a = s[i];
    const double p = (double)a.x * a.x + (double)a.y * a.y;
    if (((base + i) >> q) & 1ull) s1 += p; else s0 += p;
  }
  __shared__ double red[2][kThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
  }
  if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = s0; red[1][threadIdx.x >> 5] = s1; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double S0 = 0.0, S1 = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { S0 += red[0][w]; S1 += red[1][w]; }
    partials[(uint64_t)t * bpt + b] = make_double2(S0, S1);
  }
}

// Branch and Kraus operator of one channel on block b's share of the
// amplitude pairs of state t (every block re-reduces the state's partials
// in the same order, so all blocks take the same branch).  The uniform is
// number k of seeds[t]'s stream, or u_single when seeds is null; the branch
// goes to branch[t * branch_stride + k] when branch is not null.
__global__ void __launch_bounds__(kThreads) k_noise_apply(float2* __restrict__ states, int n, int q, int kind,
                                                          double g, int bpt, const double2* __restrict__ partials,
                                                          const uint64_t* __restrict__ seeds, double u_single,
                                                          int branch_stride, int k, uint8_t* __restrict__ branch,
                                                          int t0) {
  const int t = t0 + blockIdx.y, b = blockIdx.x;
  __shared__ double sh[2];
  if (threadIdx.x < 32) {
    double s0 = 0.0, s1 = 0.0;
    for (int j = threadIdx.x; j < bpt; j += 32) {
      const double2 v = partials[(uint64_t)t * bpt + j];
      s0 += v.x;
      s1 += v.y;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s0 += __shfl_xor_sync(0xffffffffu, s0, o);
      s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    }
    if (threadIdx.x == 0) { sh[0] = s0; sh[1] = s1; }
  }
  __syncthreads();
  const double S0 = sh[0], S1 = sh[1];
  const double p1 = g * S1 / (S0 + S1);
  const size_t slot = (size_t)t * branch_stride + k;
  const double uu = seeds ? qs_seed_uniform_at(seeds[t], (uint64_t)k) : u_single;
  // the kept branch has norm^2 keep; a branch of zero weight is never taken
  const double keep = S0 + (1.0 - g) * S1;
  const bool jump = S1 > 0.0 && (uu < p1 || !(keep > 0.0));
  if (b == 0 && threadIdx.x == 0 && branch) branch[slot] = jump ? 1 : 0;
  float f0 = 0.f, f1 = 0.f;
  if (!jump) {
    const double r = 1.0 / sqrt(keep);
    f0 = (float)r;
    f1 = (float)(sqrt(1.0 - g) * r);
  } else {
    f1 = (float)(1.0 / sqrt(S1));
  }
  const bool damp = kind == QS_OP_AMP_DAMP;
  const uint64_t N = 1ull << n, pchunk = (N >> 1) / (uint64_t)bpt;
  float2* s = states + (uint64_t)t * N;
  for (uint64_t c = (uint64_t)b * pchunk + threadIdx.x; c < (uint64_t)(b + 1) * pchunk; c += blockDim.x) {
    const uint64_t i0 = insert_zero(c, q), i1 = i0 | (1ull << q);
    const float2 a1 = s[i1];
    if (!jump) {
      const float2 a0 = s[i0];
      s[i0] = make_float2(a0.x * f0, a0.y * f0);
      s[i1] = make_float2(a1.x * f1, a1.y * f1);
    } else if (damp) {
      s[i0] = make_float2(a1.x * f1, a1.y * f1);
      s[i1] = make_float2(0.f, 0.f);
    } else {
      s[i0] = make_float2(0.f, 0.f);
      s[i1] = make_float2(a1.x * f1, a1.y * f1);
    }
  }
}

// One state-dependent channel over n_states states stored back to back;
// partials: device scratch of n_states * blocks_per_state(n) double2.
void launch_channel(qs_context* h, float2* states, int n, int n_states, int q, int kind, double g,
                    double2* partials, const uint64_t* d_seeds, double u_single, int branch_stride, int k,
                    uint8_t* d_branch) {
  const int bpt = blocks_per_state(n);
  for (int t0 = 0; t0 < n_states; t0 += 65535) {
    const int nt = std::min(65535, n_states - t0);
    dim3 grid((unsigned)bpt, (unsigned)nt);
    k_noise_sums<<<grid, kThreads, 0, h->stream>>>(states, n, q, bpt, partials, t0);
    qs_after_launch(h, "k_noise_sums");
    k_noise_apply<<<grid, kThreads, 0, h->stream>>>(states, n, q, kind, g, bpt, partials, d_seeds, u_single,
                                                    branch_stride, k, d_branch, t0);
    qs_after_launch(h, "k_noise_apply");
  }
}

void check_prob(double p, const char* what) {
  if (!(p >= 0.0 && p <= 1.0)) throw qs_error(QS_ERR_INVALID, std::string(what) + " must be in [0, 1]");
}

void single_channel(qs_context* h, void* state, int n, int target, int kind, double g, double u, int32_t* branch) {
  qs_check_state(state, n);
  qs_check_qubit(target, n, "target");
  check_prob(g, kind == QS_OP_AMP_DAMP ? "gamma" : "lambda");
  QS_CHECK_ARG(std::isfinite(u), "random value must be finite");
  const int bpt = blocks_per_state(n);
  // handle scratch: the partials, then the branch byte
  const size_t boff = (size_t)bpt * sizeof(double2);
  char* base = static_cast<char*>(h->scratch_get(boff + 16));
  uint8_t* d_branch = reinterpret_cast<uint8_t*>(base + boff);
  launch_channel(h, (float2*)state, n, 1, target, kind, g, reinterpret_cast<double2*>(base), nullptr, u, 0, 0,
                 d_branch);
  if (branch) {
    double* pin = h->pinned_get(sizeof(double));
    QS_CUDA(cudaMemcpyAsync(pin, d_branch, 1, cudaMemcpyDeviceToHost, h->stream));
    QS_CUDA(cudaStreamSynchronize(h->stream));
    *branch = (int32_t)reinterpret_cast<const uint8_t*>(pin)[0];
  }
}

// ------------------------------------------------------- trajectories ----
struct NoiseSite {
  int op;      // index in the circuit
  int kind;    // QS_OP_DEPOLARIZE / AMP_DAMP / DEPHASE
  int q;
  double p;
};

qs_op pauli_op(int q, int b) {
  qs_op o;
  std::memset(&o, 0, sizeof(o));
  o.nq = 1;
  o.q[0] = q;
  o.param = -1;
  if (b == 1) o.kind = QS_OP_MCX;
  else if (b == 2) o.kind = QS_OP_Y;
  else { o.kind = QS_OP_MCPHASE; o.m[0] = -1.0; }  // exact negation of |1>
  return o;
}

// Appends the passes of whole-state plans to a merged program, with noise
// blocks between segments; flushes a DevPass record whenever the coefficient
// pool would outgrow shared memory.
struct Merger {
  int n = 0, R = 0;
  size_t coef_cap = 0;  // float2 entries per merged pass
  std::vector<DevBlock> blocks;
  std::vector<DevOp> ops;
  std::vector<float> coef;
  int has2 = 0;
  qs_plan_s out;

  // force: emit even an empty pass (a program whose channels all came out
  // as the identity still has to write |0..0>)
  void flush(bool force = false) {
    if (blocks.empty() && !(force && out.pass_offsets.empty())) return;
    auto a16 = [](size_t x) { return (x + 15) & ~size_t(15); };
    DevPass hdr;
    std::memset(&hdr, 0, sizeof(hdr));
    hdr.T = n;
    hdr.R = R;
    hdr.nblocks = (int32_t)blocks.size();
    hdr.n_qubits = n;
    for (int k = 0; k < n; ++k) hdr.S[k] = k;
    hdr.ncoef = (uint32_t)(coef.size() / 2);
    hdr.has2 = (uint32_t)has2;
    size_t off = a16(sizeof(DevPass));
    hdr.block_off = (uint32_t)off;
    off = a16(off + blocks.size() * sizeof(DevBlock));
    hdr.op_off = (uint32_t)off;
    off = a16(off + ops.size() * sizeof(DevOp));
    hdr.coef_off = (uint32_t)off;
    off = a16(off + coef.size() * sizeof(float));
    hdr.bytes = (uint32_t)off;
    const size_t at = out.blob.size();
    out.blob.resize(at + off, 0);
    char* b = out.blob.data() + at;
    std::memcpy(b, &hdr, sizeof(hdr));
    if (!blocks.empty()) std::memcpy(b + hdr.block_off, blocks.data(), blocks.size() * sizeof(DevBlock));
    if (!ops.empty()) std::memcpy(b + hdr.op_off, ops.data(), ops.size() * sizeof(DevOp));
    if (!coef.empty()) std::memcpy(b + hdr.coef_off, coef.data(), coef.size() * sizeof(float));
    out.pass_offsets.push_back((uint32_t)at);
    out.pass_T.push_back(n);
    out.pass_R.push_back(R);
    out.pass_has2.push_back(has2);
    out.pass_ncoef.push_back((int)hdr.ncoef);
    blocks.clear();
    ops.clear();
    coef.clear();
    has2 = 0;
  }

  void add_plan(const qs_plan_s& p) {
    for (size_t j = 0; j < p.pass_offsets.size(); ++j) {
      const char* base = p.blob.data() + p.pass_offsets[j];
      DevPass hdr;
      std::memcpy(&hdr, base, sizeof(hdr));
      if (hdr.T != n || hdr.R != R) throw qs_error(QS_ERR_INVALID, "internal: noise program pass shape");
      const auto* pb = reinterpret_cast<const DevBlock*>(base + hdr.block_off);
      const auto* po = reinterpret_cast<const DevOp*>(base + hdr.op_off);
      const auto* pc = reinterpret_cast<const float*>(base + hdr.coef_off);
      int nops = 0;
      for (int b = 0; b < hdr.nblocks; ++b) nops = std::max(nops, (int)pb[b].op_end);
      if (!blocks.empty() && coef.size() / 2 + hdr.ncoef > coef_cap) flush();
      if (hdr.ncoef > coef_cap) throw qs_error(QS_ERR_INVALID, "noise program pass too large for shared memory");
      const int32_t ob = (int32_t)ops.size();
      const uint32_t cb = (uint32_t)(coef.size() / 2);
      for (int b = 0; b < hdr.nblocks; ++b) {
        DevBlock d = pb[b];
        d.op_begin += ob;
        d.op_end += ob;
        blocks.push_back(d);
      }
      for (int o = 0; o < nops; ++o) {
        DevOp d = po[o];
        d.coef += cb;
        ops.push_back(d);
      }
      coef.insert(coef.end(), pc, pc + 2 * (size_t)hdr.ncoef);
      has2 |= hdr.has2 ? 1 : 0;  // a merged program is never dense-4x4 only
    }
  }

  // One noise block for a run of consecutive channels (site index, site)
  // on at most 4 distinct qubits.
  void add_noise_group(const std::vector<std::pair<int, NoiseSite>>& group) {
    DevBlock b;
    std::memset(&b, 0, sizeof(b));
    std::vector<int> qs;
    for (const auto& e : group)
      if (std::find(qs.begin(), qs.end(), e.second.q) == qs.end()) qs.push_back(e.second.q);
    std::sort(qs.begin(), qs.end());  // the kernel inserts zeros at Q in ascending order
    const int nq = (int)qs.size();
    for (int j = 0; j < nq; ++j) b.pos[j] = (int8_t)qs[j];
    b.pos[5] = (int8_t)nq;
    b.pos[6] = 1;
    b.op_begin = (int32_t)ops.size();
    for (const auto& e : group) {
      DevOp d;
      std::memset(&d, 0, sizeof(d));
      d.kind = DK_NOISE;
      d.t0 = (uint8_t)e.second.q;
      d.d0 = (uint8_t)e.second.kind;
      d.coef = (uint32_t)e.first;
      std::memcpy(&d.gc, &e.second.p, sizeof(double));
      ops.push_back(d);
    }
    b.op_end = (int32_t)ops.size();
    blocks.push_back(b);
  }
};

// The circuit's op stream cut into unitary segments; seg_site[s] is the
// site that follows segment s.  With br (a depolarizing outcome pattern),
// each depolarizing site becomes its Pauli (or nothing) and only the
// state-dependent sites cut; without it every site cuts.
void segment_stream(const qs_op* ops, int nops, const std::vector<NoiseSite>& sites, const std::vector<uint8_t>* br,
                    std::vector<std::vector<qs_op>>& seg_ops, std::vector<int>& seg_site) {
  seg_ops.assign(1, {});
  seg_site.clear();
  size_t k = 0;
  for (int i = 0; i < nops; ++i) {
    if (k < sites.size() && sites[k].op == i) {
      const NoiseSite& s = sites[k];
      if (br && s.kind == QS_OP_DEPOLARIZE) {
        const uint8_t b = (*br)[k];
        if (b) seg_ops.back().push_back(pauli_op(s.q, b));
      } else {
        seg_site.push_back((int)k);
        seg_ops.emplace_back();
      }
      ++k;
      continue;
    }
    seg_ops.back().push_back(ops[i]);
  }
}

// The noise channels of a circuit, in program order (checked).
std::vector<NoiseSite> noise_sites(int n, const qs_op* ops, int nops) {
  std::vector<NoiseSite> sites;
  for (int i = 0; i < nops; ++i) {
    if (!is_noise(ops[i].kind)) continue;
    QS_CHECK_ARG(ops[i].nq == 1, "a noise channel acts on one qubit");
    qs_check_qubit(ops[i].q[0], n, "noise");
    check_prob(ops[i].m[0], "noise channel parameter");
    sites.push_back(NoiseSite{i, ops[i].kind, ops[i].q[0], ops[i].m[0]});
  }
  return sites;
}

// The program of a noisy circuit on up to 14 qubits: its unitary segments
// planned as whole-state passes, consecutive channels grouped into noise
// blocks between them.  auto_bb: the block width was not fixed by the caller.
qs_plan_s whole_state_program(int n, const qs_op* ops, int nops, const std::vector<NoiseSite>& sites, int tb, int bb,
                              bool auto_bb) {
  std::vector<std::vector<qs_op>> seg;
  std::vector<int> seg_site;
  segment_stream(ops, nops, sites, nullptr, seg, seg_site);
  // channels after (almost) every gate leave segments of one or two gates:
  // 3-qubit register blocks then beat wider ones (smaller diagonal tables,
  // so more CTAs per SM; measured 204 k vs 182 k trajectories/s on a
  // 12-qubit, 840-channel circuit)
  {
    size_t nonempty = 0, gates = 0;
    for (const auto& sg : seg) {
      nonempty += !sg.empty();
      gates += sg.size();
    }
    if (auto_bb && nonempty && gates <= 4 * nonempty) bb = std::min(bb, 3);
  }
  const size_t smem_left = 200 * 1024 - (8ull << n) - 2 * 128 * sizeof(uint64_t) - 16 * sizeof(int) - 16;
  Merger m;
  m.n = n;
  m.R = std::min(bb, n);
  m.coef_cap = std::min<size_t>(8192, smem_left / sizeof(float2));
  m.out.n_qubits = n;
  double flops = 0;
  // consecutive channels (no gate between) share a block while they touch
  // at most kGroupQubits qubits and number at most kGroupOps
  constexpr int kGroupQubits = 4, kGroupOps = 32;
  std::vector<std::pair<int, NoiseSite>> group;
  auto group_qubits = [&](int extra) {
    std::vector<int> qs;
    for (const auto& e : group)
      if (std::find(qs.begin(), qs.end(), e.second.q) == qs.end()) qs.push_back(e.second.q);
    if (extra >= 0 && std::find(qs.begin(), qs.end(), extra) == qs.end()) qs.push_back(extra);
    return (int)qs.size();
  };
  auto flush_group = [&]() {
    if (!group.empty()) m.add_noise_group(group);
    group.clear();
  };
  for (size_t s = 0; s < seg.size(); ++s) {
    if (!seg[s].empty()) {
      flush_group();
      qs_plan_s p;
      qs_build_plan(n, seg[s].data(), (int)seg[s].size(), tb, &p, bb);
      m.add_plan(p);
      flops += p.info.flops;
    }
    if (s < seg_site.size()) {
      const NoiseSite& ns = sites[seg_site[s]];
      if ((int)group.size() >= kGroupOps || group_qubits(ns.q) > kGroupQubits) flush_group();
      group.emplace_back(seg_site[s], ns);
    }
  }
  flush_group();
  m.flush(true);
  m.out.info.flops = flops;
  return std::move(m.out);
}

}  // namespace

extern "C" {

int qs_apply_depolarizing(qs_handle_t h, void* state, int n, int target, double p, double u, int32_t* branch) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  qs_check_state(state, n);
  qs_check_qubit(target, n, "target");
  check_prob(p, "p");
  QS_CHECK_ARG(std::isfinite(u), "random value must be finite");
  const int b = qs_depol_branch(p, u);
  if (b) {
    const uint64_t npairs = 1ull << (n - 1);
    const int grid = qs_blocks_for(h, npairs, kThreads);
    k_pauli<<<grid, kThreads, 0, h->stream>>>((float2*)state, target, b, npairs);
    qs_after_launch(h, "k_pauli");
  }
  if (branch) *branch = b;
  QS_API_END(h)
}

int qs_apply_amplitude_damping(qs_handle_t h, void* state, int n, int target, double gamma, double u,
                               int32_t* branch) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  single_channel(h, state, n, target, QS_OP_AMP_DAMP, gamma, u, branch);
  QS_API_END(h)
}

int qs_apply_dephasing(qs_handle_t h, void* state, int n, int target, double lambda, double u, int32_t* branch) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  single_channel(h, state, n, target, QS_OP_DEPHASE, lambda, u, branch);
  QS_API_END(h)
}

int qs_noise_program(int n, const qs_op* ops, int nops, int block_bits, void* out, size_t cap, size_t* needed) {
  qs_context* h = nullptr;
  QS_API_BEGIN
  QS_CHECK_ARG(needed != nullptr, "needed is null");
  QS_CHECK_ARG(n >= 1 && n <= 14, "whole-state noise programs hold 1 to 14 qubits");
  QS_CHECK_ARG(nops >= 0 && (nops == 0 || ops), "ops pointer is null");
  QS_CHECK_ARG(block_bits == 0 || (block_bits >= 2 && block_bits <= 5), "block_bits must be 0 (auto) or in [2, 5]");
  const std::vector<NoiseSite> sites = noise_sites(n, ops, nops);
  const qs_plan_s p = whole_state_program(n, ops, nops, sites, 13, block_bits ? block_bits : 4, block_bits == 0);
  *needed = p.blob.size();
  if (out && cap >= p.blob.size() && !p.blob.empty()) std::memcpy(out, p.blob.data(), p.blob.size());
  QS_API_END(h)
}

int qs_noise_trajectories(qs_handle_t h, int n, const qs_op* ops, int nops, int n_traj, const uint64_t* seeds,
                          void* states, uint8_t* branches_host) {
  QS_REQUIRE_HANDLE(h);
  uint64_t* d_seeds = nullptr;
  uint8_t* d_br = nullptr;
  qs_batch_plan_s* B = nullptr;
  try {
  qs_check_state(states, n);
  QS_CHECK_ARG(n_traj >= 0, "n_traj must be >= 0");
  QS_CHECK_ARG(nops >= 0 && (nops == 0 || ops), "ops pointer is null");
  QS_CHECK_ARG(n_traj == 0 || seeds, "seeds pointer is null");
  if (n_traj == 0) return QS_OK;
  const std::vector<NoiseSite> sites = noise_sites(n, ops, nops);
  const int nn = (int)sites.size();
  const bool want_br = branches_host && nn;
  const size_t slots = (size_t)n_traj * (size_t)nn;
  if (want_br) QS_CUDA(cudaMallocAsync((void**)&d_br, slots, h->stream));
  const uint64_t N = 1ull << n;
  int tb = 0, bb = 0;
  qs_plan_shape(h, n, false, tb, bb);

  if (n <= 14) {
    // one whole-state program with a noise block per channel group, shared
    // by all trajectories; one CTA per trajectory
    std::vector<qs_plan_s> progs(1);
    progs[0] = whole_state_program(n, ops, nops, sites, tb, bb, h->block_bits == 0);
    std::vector<BatchUnit> units(n_traj);
    for (int t = 0; t < n_traj; ++t)
      units[t] = BatchUnit{0, (uint64_t)t * N, seeds[t], want_br ? d_br + (size_t)t * nn : nullptr};
    B = qs_batch_build_units(h, progs, units, true, noise_threads());
    qs_batch_launch(h, B, states);
    qs_batch_release(B);
    B = nullptr;
  } else {
    // depolarizing outcomes on the host; trajectories with the same outcomes
    // share their segment programs
    std::vector<uint8_t> Br(want_br ? slots : 0, 0);
    std::map<std::vector<uint8_t>, int> pattern_id;
    std::vector<std::vector<uint8_t>> patterns;
    std::vector<int> traj_pattern(n_traj);
    for (int t = 0; t < n_traj; ++t) {
      std::vector<uint8_t> key(nn, 0);
      for (int k = 0; k < nn; ++k)
        if (sites[k].kind == QS_OP_DEPOLARIZE) {
          key[k] = (uint8_t)qs_depol_branch(sites[k].p, qs_seed_uniform_at(seeds[t], (uint64_t)k));
          if (want_br) Br[(size_t)t * nn + k] = key[k];
        }
      auto it = pattern_id.find(key);
      if (it == pattern_id.end()) {
        it = pattern_id.emplace(key, (int)patterns.size()).first;
        patterns.push_back(key);
      }
      traj_pattern[t] = it->second;
    }
    if (want_br) QS_CUDA(cudaMemcpyAsync(d_br, Br.data(), slots, cudaMemcpyHostToDevice, h->stream));
    std::vector<std::vector<std::vector<qs_op>>> seg_of(patterns.size());
    std::vector<int> seg_site;
    for (size_t pi = 0; pi < patterns.size(); ++pi)
      segment_stream(ops, nops, sites, &patterns[pi], seg_of[pi], seg_site);
    const size_t nseg = seg_site.size() + 1;
    bool need_init = false;
    for (int t = 0; t < n_traj; ++t) need_init |= seg_of[traj_pattern[t]][0].empty();
    if (need_init && qs_state_init_batched(h, states, n_traj, n) != QS_OK) throw qs_error(QS_ERR_CUDA, h->err);
    double2* partials = nullptr;
    if (!seg_site.empty()) {
      QS_CUDA(cudaMallocAsync((void**)&d_seeds, (size_t)n_traj * sizeof(uint64_t), h->stream));
      QS_CUDA(cudaMemcpyAsync(d_seeds, seeds, (size_t)n_traj * sizeof(uint64_t), cudaMemcpyHostToDevice,
                              h->stream));
      partials = static_cast<double2*>(h->scratch_get((size_t)n_traj * blocks_per_state(n) * sizeof(double2)));
    }
    for (size_t s = 0; s < nseg; ++s) {
      std::map<std::vector<uint8_t>, int> seg_plan;  // outcomes within the segment -> plan
      std::vector<qs_plan_s> plans;
      std::vector<BatchUnit> units;
      std::vector<int> plan_of_pattern(patterns.size(), -1);
      const int lo = s == 0 ? -1 : seg_site[s - 1], hi = s < seg_site.size() ? seg_site[s] : nn;
      for (size_t pi = 0; pi < patterns.size(); ++pi) {
        const auto& so = seg_of[pi][s];
        if (so.empty()) continue;
        // the segment's stream is fixed by the depolarizing outcomes inside it
        std::vector<uint8_t> key;
        for (int k = lo + 1; k < hi; ++k) key.push_back(patterns[pi][k]);
        auto it = seg_plan.find(key);
        if (it == seg_plan.end()) {
          it = seg_plan.emplace(key, (int)plans.size()).first;
          plans.emplace_back();
          qs_build_plan(n, so.data(), (int)so.size(), tb, &plans.back(), bb);
        }
        plan_of_pattern[pi] = it->second;
      }
      for (int t = 0; t < n_traj; ++t) {
        const int pl = plan_of_pattern[traj_pattern[t]];
        if (pl >= 0) units.push_back(BatchUnit{pl, (uint64_t)t * N, 0, nullptr});
      }
      if (!units.empty()) {
        B = qs_batch_build_units(h, plans, units, s == 0 && !need_init);
        qs_batch_launch(h, B, states);
        qs_batch_release(B);
        B = nullptr;
      }
      if (s < seg_site.size()) {
        const NoiseSite& ns = sites[seg_site[s]];
        launch_channel(h, (float2*)states, n, n_traj, ns.q, ns.kind, ns.p, partials, d_seeds, 0.0, nn,
                       seg_site[s], d_br);
      }
    }
  }
  if (want_br) {
    QS_CUDA(cudaMemcpyAsync(branches_host, d_br, slots, cudaMemcpyDeviceToHost, h->stream));
    QS_CUDA(cudaFreeAsync(d_br, h->stream));
    d_br = nullptr;
  }
  if (d_seeds) {
    QS_CUDA(cudaFreeAsync(d_seeds, h->stream));
    d_seeds = nullptr;
  }
  if (want_br) QS_CUDA(cudaStreamSynchronize(h->stream));
  return QS_OK;
  } catch (const std::exception& e) {
    if (B) qs_batch_release(B);
    if (d_seeds) cudaFreeAsync(d_seeds, h->stream);
    if (d_br) cudaFreeAsync(d_br, h->stream);
    const qs_error* qe = dynamic_cast<const qs_error*>(&e);
    h->err = e.what();
    return qe ? qe->code : QS_ERR_INVALID;
  }
}

}  // extern "C"
