// field.cu -- the learned field of a context: geometry, sampling, exact
// labels, GPU training (forward/backward and Adam kernels), packing of the
// inference copies, validation and the exact-evaluation bitmap, and the
// ccs_field_* entry points of include/massccs_gpu.h.
//
// No counterpart in the reference (cces-cepid/massccs): its trajectory loop
// evaluates every force exactly (src/Force.cpp:34-1725).  The network learns
// the far part of the range-separated pair terms (field_device.cuh): the
// labels are those terms weighted by 1 - S(r), summed over the target's atoms
// within the cutoffs with this engine's own cell grid and parameter tables.
//
// Training is deterministic for a given seed: samples and batches come from a
// counter-based hash, the weight gradients from a fixed-order reduction, and
// the hash-table gradients are accumulated as 64-bit fixed-point integers
// (integer addition is associative, so the atomics' order does not matter).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include <cub/device/device_select.cuh>

#include "engine_ctx.h"

using namespace ccs;
using namespace ccs_internal;

namespace {

// Master MLP vector (FP32): W1 [64][32], b1 [64], W2 [64][64], b2 [64], W3 [5][64], b3 [5].
constexpr int MO_W1 = 0;
constexpr int MO_B1 = MO_W1 + FL_H * FL_E;
constexpr int MO_W2 = MO_B1 + FL_H;
constexpr int MO_B2 = MO_W2 + FL_H * FL_H;
constexpr int MO_W3 = MO_B2 + FL_H;
constexpr int MO_B3 = MO_W3 + FL_NF * FL_H;
constexpr int NM = MO_B3 + FL_NF;
constexpr double FIX_SCALE = 1099511627776.0;  // 2^40: fixed-point table gradients

struct TrainGeo {
  float lo[3];
  float scale[FL_LEVELS];
  int res[FL_LEVELS];
  int dense[FL_LEVELS];
  uint32_t tmask;
  int log2t;
  float s[FL_NF];        // output scales
  float gs[FL_NF];       // RMS gradient of each field's labels
  float u0[FL_NF], f0[FL_NF];  // loss floors of each field's value and gradient
};

// What a field is, for its labels: the far potential of a gas site type
// (LJ parameter set lj: 0 none, 1 primary, 2 carbon; charge q) or component
// a of the far electric field.
struct FieldKind {
  int kind[FL_NF];   // 0 potential, 1 field component
  int lj[FL_NF];
  double q[FL_NF];
  int comp[FL_NF];
};

uint64_t mix64(uint64_t x) {  // splitmix64 finaliser (host)
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

}  // namespace

struct FieldState {
  ccs_field_params p{};
  int nf = 1, site_field[3] = {0, 0, 0}, dip_site = -1, efield = 0;
  FieldKind kinds{};
  FieldK k{};
  TrainGeo geo{};
  double lo[3] = {0, 0, 0}, side = 0;
  double s[FL_NF] = {1, 1, 1, 1, 1}, gs[FL_NF] = {1, 1, 1, 1, 1};  // output and gradient scales
  size_t rows = 0;  // table rows per level
  size_t nwords = 0;
  // parameters and optimiser state
  float2 *table = nullptr, *tm = nullptr, *tv = nullptr;
  unsigned long long *tgrad = nullptr;
  float *mlp = nullptr, *mm = nullptr, *mv = nullptr, *mgrad = nullptr;
  // inference copies
  uint32_t *table_bf16 = nullptr;
  float *mlp_inf = nullptr;
  uint4 *umma = nullptr;
  uint32_t *bits = nullptr;
  // samples
  float4 *spos = nullptr;
  float *slab = nullptr;
  size_t nsamples = 0;
  // per-step scratch
  float *L1 = nullptr, *R1 = nullptr, *L2 = nullptr, *R2 = nullptr, *V3 = nullptr, *part = nullptr,
        *lossbuf = nullptr;
  int *bidx = nullptr;
  size_t scratch_batch = 0, part_rows = 0;
  bool ready = false;
};

namespace {

__device__ __forceinline__ uint64_t dmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
// uniform in [0, 1) from the top 24 bits
__device__ __forceinline__ float u01(uint64_t h) { return (float)(h >> 40) * (1.0f / 16777216.0f); }

// ---- exact-evaluation bitmap: voxels within radius R of an atom -------------
__global__ void bitmap_atoms_kernel(const float4 *__restrict__ atoms, int natoms, FieldK F, float vox, float R,
                                    uint32_t *bits) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= natoms) return;
  const float4 p = atoms[a];
  const float c[3] = {p.x, p.y, p.z};
  int lo[3], hi[3];
  const int dims[3] = {F.vx, F.vy, F.vz};
  for (int d = 0; d < 3; d++) {
    lo[d] = max(0, (int)floorf((c[d] - R - F.lo[d]) / vox));
    hi[d] = min(dims[d] - 1, (int)floorf((c[d] + R - F.lo[d]) / vox));
  }
  const float R2 = R * R;
  for (int k = lo[2]; k <= hi[2]; k++)
    for (int j = lo[1]; j <= hi[1]; j++)
      for (int i = lo[0]; i <= hi[0]; i++) {
        const float dx = F.lo[0] + (i + 0.5f) * vox - c[0];
        const float dy = F.lo[1] + (j + 0.5f) * vox - c[1];
        const float dz = F.lo[2] + (k + 0.5f) * vox - c[2];
        if (dx * dx + dy * dy + dz * dz < R2) {
          const uint32_t v = (uint32_t)i + (uint32_t)F.vx * ((uint32_t)j + (uint32_t)F.vy * (uint32_t)k);
          atomicOr(&bits[v >> 5], 1u << (v & 31u));
        }
      }
}

// ---- samples: candidates (uniform in the domain, or in the shell around a
// random atom), kept where the field is used (not flagged) -------------------
__global__ void sample_kernel(uint64_t seed, uint64_t first, size_t n, const float4 *__restrict__ atoms, int natoms,
                              FieldK F, float near_frac, float r_in, float shell, float4 *out, char *keep) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t base = dmix64(seed ^ dmix64(first + i));
  float x, y, z;
  if (u01(dmix64(base + 1)) < near_frac) {
    const int a = (int)(dmix64(base + 2) % (uint64_t)natoms);
    const float4 p = atoms[a];
    const float cz = 2.f * u01(dmix64(base + 3)) - 1.f, ph = 6.28318530717958647692f * u01(dmix64(base + 4));
    const float sz = sqrtf(fmaxf(0.f, 1.f - cz * cz));
    const float r = r_in + shell * u01(dmix64(base + 5));
    x = p.x + r * sz * cosf(ph);
    y = p.y + r * sz * sinf(ph);
    z = p.z + r * cz;
  } else {
    x = F.lo[0] + F.side * u01(dmix64(base + 6));
    y = F.lo[1] + F.side * u01(dmix64(base + 7));
    z = F.lo[2] + F.side * u01(dmix64(base + 8));
  }
  out[i] = make_float4(x, y, z, 0.f);
  keep[i] = field_exact(F, x, y, z) ? 0 : 1;
}

// Far-part labels (value and minus the gradient of every field) at n
// points: one warp per point, lanes over the (x, y) columns of the cell grid
// that meet the reach sphere, FP64 sums of the FP32 pair terms.
__global__ void __launch_bounds__(256) far_label_kernel(KParams kp, FieldKind fk, int nf, size_t n,
                                                        const float4 *__restrict__ pos, float *lab) {
  const int lane = threadIdx.x & 31;
  const size_t w = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
  const float rin = kp.field.r_in, rout = kp.field.r_out;
  const float rlj2 = (float)kp.rlj2, rc2 = (float)kp.rc2;
  for (size_t i = w; i < n; i += nw) {
    const float4 P = pos[i];
    double acc[FL_NF][4];
#pragma unroll
    for (int f = 0; f < FL_NF; f++) acc[f][0] = acc[f][1] = acc[f][2] = acc[f][3] = 0.0;
    const float R = (float)kp.reach + 1e-3f;
    int i0, j0, nj;
    float inv_nj;
    const int ncol = column_range<float>(kp, P.x, P.y, R, i0, j0, nj, inv_nj);
    for (int c = lane; c < ncol; c += 32) {
      int b, len;
      column_run<float>(kp, c, ncol, i0, j0, nj, inv_nj, P.x, P.y, P.z, R, b, len);
      for (int ai = b; ai < b + len; ai++) {
        const float4 a = __ldg(&kp.xyzq32[ai]);
        const float dx = P.x - a.x, dy = P.y - a.y, dz = P.z - a.z;
        const float r2 = dx * dx + dy * dy + dz * dz;
        const float ir = rsqrtf(r2), ir2 = ir * ir, ir3 = ir * ir2;
        float S, dS;
        range_switch(r2 * ir, rin, rout, S, dS);
        const float wf = 1.f - S, dsr = dS * ir;  // far weight; S'(r) / r
        const bool in_lj = r2 < rlj2, in_c = r2 < rc2;
        for (int f = 0; f < nf; f++) {
          if (fk.kind[f] == 0) {  // far potential: (1 - S) u, force (1 - S) F + u S' d / r
            float u = 0.f, fs = 0.f;
            if (fk.lj[f]) {
              const float2 ab = __ldg(fk.lj[f] == 2 ? &kp.abc32[ai] : &kp.ab32[ai]);
              const float ir6 = ir2 * ir2 * ir2;
              if (in_lj) {
                u += ir6 * (ab.x * ir6 - ab.y) - (ab.x * (float)kp.rc12inv - ab.y * (float)kp.rc6inv);
                fs += ir6 * (12.f * ab.x * ir6 - 6.f * ab.y) * ir2;
              }
            }
            if (fk.q[f] != 0.0 && kp.coul_on && in_c) {
              const float kq = (float)(KCOUL * fk.q[f]) * a.w;
              u += kq * (ir - (float)kp.c1 + (float)kp.c2 * r2);
              fs += kq * (ir3 - (float)kp.rc3inv);
            }
            const float fsc = wf * fs + u * dsr;
            acc[f][0] += (double)(wf * u);
            acc[f][1] += (double)(fsc * dx); acc[f][2] += (double)(fsc * dy); acc[f][3] += (double)(fsc * dz);
          } else if (in_c) {  // far field component a: (1 - S) e_a, minus its gradient
            const int ca = fk.comp[f];
            const float sq = a.w * (ir3 - (float)kp.rc3inv), tq = -3.f * a.w * ir3 * ir2;
            const float d[3] = {dx, dy, dz};
            acc[f][0] += (double)(wf * sq * d[ca]);
            // grad (1 - S) e_a = (1 - S)(sq delta_a + tq d_a d) - sq d_a (S'/r) d
            const float t2 = wf * tq * d[ca] - sq * d[ca] * dsr;
#pragma unroll
            for (int b = 0; b < 3; b++) acc[f][1 + b] -= (double)(t2 * d[b] + (b == ca ? wf * sq : 0.f));
          }
        }
      }
    }
#pragma unroll
    for (int f = 0; f < FL_NF; f++)
#pragma unroll
      for (int k = 0; k < 4; k++)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc[f][k] += __shfl_xor_sync(0xffffffffu, acc[f][k], o);
    if (lane == 0)
      for (int f = 0; f < nf; f++)
        for (int k = 0; k < 4; k++) lab[(i * nf + f) * 4 + k] = (float)acc[f][k];
  }
}

// batch indices of a training step (with replacement, counter-based)
__global__ void batch_kernel(uint64_t seed, uint64_t step, int B, size_t n, int *bidx) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= B) return;
  bidx[j] = (int)(dmix64(seed ^ dmix64((step << 32) + (uint64_t)j + 0x5bd1e995ull)) % (uint64_t)n);
}

// ---- training forward/backward: one warp per sample --------------------------
// Lane l: encoded feature l (level l >> 1) with its Jacobian row, hidden
// units 2l and 2l + 1, corners 4 (l & 1) .. + 3 of its level.  Writes the
// outer-product factors of the weight gradients (pairs p = 0: potential
// path, p = 1 + f: force path of field f), the output-layer gradient terms,
// the sample's loss, and adds the table gradients (fixed point).
template <int NF>
__global__ void __launch_bounds__(256) train_kernel(const float2 *__restrict__ table, const float *__restrict__ mlp,
                                                    TrainGeo G, const float4 *__restrict__ pos,
                                                    const float *__restrict__ lab, const int *__restrict__ bidx,
                                                    int B, float lam_u, float invB, float *L1,
                                                    float *R1, float *L2, float *R2, float *V3, float *lossbuf,
                                                    unsigned long long *tgrad) {
  constexpr int P = 1 + NF;
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ float smw[];
  float *sW1 = smw, *sW1t = sW1 + FL_H * FL_E, *sW2 = sW1t + FL_E * FL_H, *sW2t = sW2 + FL_H * FL_H;
  float *sb1 = sW2t + FL_H * FL_H, *sb2 = sb1 + FL_H, *sw3 = sb2 + FL_H, *sb3 = sw3 + FL_NF * FL_H;
  for (int t = threadIdx.x; t < FL_H * FL_E; t += blockDim.x) {
    const float w = mlp[MO_W1 + t];
    sW1[t] = w;
    sW1t[(t % FL_E) * FL_H + t / FL_E] = w;
  }
  for (int t = threadIdx.x; t < FL_H * FL_H; t += blockDim.x) {
    const float w = mlp[MO_W2 + t];
    sW2[t] = w;
    sW2t[(t % FL_H) * FL_H + t / FL_H] = w;
  }
  for (int t = threadIdx.x; t < FL_H; t += blockDim.x) { sb1[t] = mlp[MO_B1 + t]; sb2[t] = mlp[MO_B2 + t]; }
  for (int t = threadIdx.x; t < FL_NF * FL_H; t += blockDim.x) sw3[t] = mlp[MO_W3 + t];
  if (threadIdx.x < FL_NF) sb3[threadIdx.x] = mlp[MO_B3 + threadIdx.x];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int lev = lane >> 1, half = lane & 1;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int j = gw; j < B; j += nw) {
    const int si = bidx[j];
    const float4 p4 = pos[si];
    const float x[3] = {p4.x, p4.y, p4.z};
    // ---- encoding (FP32 table)
    int c0[3];
    float S[3], dS[3];
    {
      const float sc = G.scale[lev];
      const int r = G.res[lev];
#pragma unroll
      for (int a = 0; a < 3; a++) {
        const float pp = fminf(fmaxf((x[a] - G.lo[a]) * sc, 0.f), (float)r);
        const int c = min((int)floorf(pp), r - 1);
        const float f = pp - (float)c;
        c0[a] = c;
        S[a] = f * f * (3.f - 2.f * f);
        dS[a] = 6.f * f * (1.f - f) * sc;
      }
    }
    uint32_t rows[4];
    float w[4], dw[4][3];
    float e0 = 0.f, e1 = 0.f, j0[3] = {0.f, 0.f, 0.f}, j1[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int cc = 0; cc < 4; cc++) {
      const int c = 4 * half + cc;
      const int ox = c & 1, oy = (c >> 1) & 1, oz = (c >> 2) & 1;
      const float wx = ox ? S[0] : 1.f - S[0], wy = oy ? S[1] : 1.f - S[1], wz = oz ? S[2] : 1.f - S[2];
      const float dx = ox ? dS[0] : -dS[0], dy = oy ? dS[1] : -dS[1], dz = oz ? dS[2] : -dS[2];
      const int cx = c0[0] + ox, cy = c0[1] + oy, cz = c0[2] + oz;
      uint32_t row;
      if (G.dense[lev]) {
        const uint32_t rr = (uint32_t)G.res[lev] + 1u;
        row = (uint32_t)cx + rr * ((uint32_t)cy + rr * (uint32_t)cz);
      } else {
        row = ((uint32_t)cx * 1u ^ (uint32_t)cy * 2654435761u ^ (uint32_t)cz * 805459861u) & G.tmask;
      }
      rows[cc] = row;
      const float2 t = table[((size_t)lev << G.log2t) + row];
      w[cc] = wx * wy * wz;
      dw[cc][0] = dx * wy * wz; dw[cc][1] = wx * dy * wz; dw[cc][2] = wx * wy * dz;
      e0 += w[cc] * t.x; e1 += w[cc] * t.y;
#pragma unroll
      for (int a = 0; a < 3; a++) { j0[a] += dw[cc][a] * t.x; j1[a] += dw[cc][a] * t.y; }
    }
    e0 += __shfl_xor_sync(FULL, e0, 1);
    e1 += __shfl_xor_sync(FULL, e1, 1);
#pragma unroll
    for (int a = 0; a < 3; a++) {
      j0[a] += __shfl_xor_sync(FULL, j0[a], 1);
      j1[a] += __shfl_xor_sync(FULL, j1[a], 1);
    }
    const float ek = half ? e1 : e0;
    const float Jk[3] = {half ? j1[0] : j0[0], half ? j1[1] : j0[1], half ? j1[2] : j0[2]};
    const int u0i = 2 * lane, u1i = 2 * lane + 1;  // this lane's hidden units
    // ---- forward
    float z1a = sb1[u0i], z1b = sb1[u1i];
#pragma unroll 8
    for (int k = 0; k < FL_E; k++) {
      const float xk = __shfl_sync(FULL, ek, k);
      z1a += sW1t[k * FL_H + u0i] * xk; z1b += sW1t[k * FL_H + u1i] * xk;
    }
    const bool m1a = z1a > 0.f, m1b = z1b > 0.f;
    const float a1a = m1a ? z1a : 0.f, a1b = m1b ? z1b : 0.f;
    float z2a = sb2[u0i], z2b = sb2[u1i];
#pragma unroll 8
    for (int jj = 0; jj < FL_H; jj++) {
      const float aj = __shfl_sync(FULL, (jj & 1) ? a1b : a1a, jj >> 1);
      z2a += sW2t[jj * FL_H + u0i] * aj; z2b += sW2t[jj * FL_H + u1i] * aj;
    }
    const bool m2a = z2a > 0.f, m2b = z2b > 0.f;
    const float a2a = m2a ? z2a : 0.f, a2b = m2b ? z2b : 0.f;
    // ---- per field: potential, force, loss terms
    const float *lb = lab + (size_t)si * NF * 4;
    float du[NF], eF[NF][3], g0[NF], g1a[NF], g1b[NF], g2a[NF], g2b[NF];
    float loss = 0.f;
#pragma unroll
    for (int f = 0; f < NF; f++) {
      float up = sw3[f * FL_H + u0i] * a2a + sw3[f * FL_H + u1i] * a2b;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) up += __shfl_xor_sync(FULL, up, o);
      const float u = G.s[f] * (up + sb3[f]);
      g2a[f] = m2a ? sw3[f * FL_H + u0i] : 0.f;
      g2b[f] = m2b ? sw3[f * FL_H + u1i] : 0.f;
      float ga = 0.f, gb = 0.f;
#pragma unroll 8
      for (int o = 0; o < FL_H; o++) {
        const float go = __shfl_sync(FULL, (o & 1) ? g2b[f] : g2a[f], o >> 1);
        ga += sW2[o * FL_H + u0i] * go; gb += sW2[o * FL_H + u1i] * go;
      }
      g1a[f] = m1a ? ga : 0.f;
      g1b[f] = m1b ? gb : 0.f;
      float g = 0.f;
#pragma unroll 8
      for (int i = 0; i < FL_H; i++) {
        const float gi = __shfl_sync(FULL, (i & 1) ? g1b[f] : g1a[f], i >> 1);
        g += sW1[i * FL_E + lane] * gi;
      }
      g0[f] = g;
      float Fv[3] = {g * Jk[0], g * Jk[1], g * Jk[2]};
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int a = 0; a < 3; a++) Fv[a] += __shfl_xor_sync(FULL, Fv[a], o);
      }
      const float U = lb[4 * f], Fs[3] = {lb[4 * f + 1], lb[4 * f + 2], lb[4 * f + 3]};
      const float wu = lam_u / (U * U + G.u0[f] * G.u0[f]);
      const float wf = 1.f / (Fs[0] * Fs[0] + Fs[1] * Fs[1] + Fs[2] * Fs[2] + G.f0[f] * G.f0[f]);
      const float d = u - U;
      du[f] = 2.f * wu * d * invB;
      float fl = 0.f;
#pragma unroll
      for (int a = 0; a < 3; a++) {
        const float dF = -G.s[f] * Fv[a] - Fs[a];
        eF[f][a] = 2.f * wf * dF * invB;
        fl += dF * dF;
      }
      loss += wu * d * d + wf * fl;
    }
    // ---- potential path backward
    float da2a = 0.f, da2b = 0.f;
#pragma unroll
    for (int f = 0; f < NF; f++) {
      da2a += G.s[f] * du[f] * sw3[f * FL_H + u0i];
      da2b += G.s[f] * du[f] * sw3[f * FL_H + u1i];
    }
    const float dz2a = m2a ? da2a : 0.f, dz2b = m2b ? da2b : 0.f;
    float da1a = 0.f, da1b = 0.f;
#pragma unroll 8
    for (int i = 0; i < FL_H; i++) {
      const float di = __shfl_sync(FULL, (i & 1) ? dz2b : dz2a, i >> 1);
      da1a += sW2[i * FL_H + u0i] * di; da1b += sW2[i * FL_H + u1i] * di;
    }
    const float dz1a = m1a ? da1a : 0.f, dz1b = m1b ? da1b : 0.f;
    float de = 0.f;
#pragma unroll 8
    for (int i = 0; i < FL_H; i++) {
      const float di = __shfl_sync(FULL, (i & 1) ? dz1b : dz1a, i >> 1);
      de += sW1[i * FL_E + lane] * di;
    }
    const size_t rp = (size_t)j * P;
    reinterpret_cast<float2 *>(L1 + rp * FL_H)[lane] = make_float2(dz1a, dz1b);
    R1[rp * FL_E + lane] = ek;
    reinterpret_cast<float2 *>(L2 + rp * FL_H)[lane] = make_float2(dz2a, dz2b);
    reinterpret_cast<float2 *>(R2 + rp * FL_H)[lane] = make_float2(a1a, a1b);
    // ---- force paths
    float dJ[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int f = 0; f < NF; f++) {
      const float r0 = -G.s[f] * (Jk[0] * eF[f][0] + Jk[1] * eF[f][1] + Jk[2] * eF[f][2]);
#pragma unroll
      for (int a = 0; a < 3; a++) dJ[a] += -G.s[f] * g0[f] * eF[f][a];
      float r1a = 0.f, r1b = 0.f;
#pragma unroll 8
      for (int k = 0; k < FL_E; k++) {
        const float rk = __shfl_sync(FULL, r0, k);
        r1a += sW1t[k * FL_H + u0i] * rk; r1b += sW1t[k * FL_H + u1i] * rk;
      }
      const float ha = m1a ? r1a : 0.f, hb = m1b ? r1b : 0.f;
      float r2a = 0.f, r2b = 0.f;
#pragma unroll 8
      for (int i = 0; i < FL_H; i++) {
        const float hi = __shfl_sync(FULL, (i & 1) ? hb : ha, i >> 1);
        r2a += sW2t[i * FL_H + u0i] * hi; r2b += sW2t[i * FL_H + u1i] * hi;
      }
      const size_t rf = rp + 1 + f;
      reinterpret_cast<float2 *>(L1 + rf * FL_H)[lane] = make_float2(g1a[f], g1b[f]);
      R1[rf * FL_E + lane] = r0;
      reinterpret_cast<float2 *>(L2 + rf * FL_H)[lane] = make_float2(g2a[f], g2b[f]);
      reinterpret_cast<float2 *>(R2 + rf * FL_H)[lane] = make_float2(ha, hb);
      float *v3 = V3 + ((size_t)j * NF + f) * (FL_H + 1);
      v3[u0i] = G.s[f] * du[f] * a2a + (m2a ? r2a : 0.f);
      v3[u1i] = G.s[f] * du[f] * a2b + (m2b ? r2b : 0.f);
      if (lane == 0) v3[FL_H] = G.s[f] * du[f];
    }
    if (lane == 0) lossbuf[j] = loss * invB;
    // ---- table gradients of this lane's 4 corners, both features of its level
    const float deo = __shfl_xor_sync(FULL, de, 1);
    float dJo[3];
#pragma unroll
    for (int a = 0; a < 3; a++) dJo[a] = __shfl_xor_sync(FULL, dJ[a], 1);
    const float de0 = half ? deo : de, de1 = half ? de : deo;
    const float dJ0[3] = {half ? dJo[0] : dJ[0], half ? dJo[1] : dJ[1], half ? dJo[2] : dJ[2]};
    const float dJ1[3] = {half ? dJ[0] : dJo[0], half ? dJ[1] : dJo[1], half ? dJ[2] : dJo[2]};
#pragma unroll
    for (int cc = 0; cc < 4; cc++) {
      const float ga = w[cc] * de0 + dw[cc][0] * dJ0[0] + dw[cc][1] * dJ0[1] + dw[cc][2] * dJ0[2];
      const float gb = w[cc] * de1 + dw[cc][0] * dJ1[0] + dw[cc][1] * dJ1[1] + dw[cc][2] * dJ1[2];
      unsigned long long *tg = tgrad + 2 * (((size_t)lev << G.log2t) + rows[cc]);
      if (ga != 0.f) atomicAdd(&tg[0], (unsigned long long)__double2ll_rn((double)ga * FIX_SCALE));
      if (gb != 0.f) atomicAdd(&tg[1], (unsigned long long)__double2ll_rn((double)gb * FIX_SCALE));
    }
  }
}

// ---- weight gradients: fixed-order reduction of the per-sample factors -----
constexpr int WG_CH = 512;  // samples per CTA
template <int NF>
__global__ void __launch_bounds__(256) wgrad_kernel(const float *__restrict__ L1, const float *__restrict__ R1,
                                                    const float *__restrict__ L2, const float *__restrict__ R2,
                                                    const float *__restrict__ V3, int B, float *part) {
  constexpr int P = 1 + NF;
  constexpr int TR = 16;
  __shared__ float sL1[TR][FL_H], sR1[TR][FL_E], sL2[TR][FL_H], sR2[TR][FL_H];
  const int t = threadIdx.x;
  const int jb = blockIdx.x * WG_CH, je = min(B, jb + WG_CH);
  const size_t r0 = (size_t)jb * P, r1 = (size_t)je * P;
  float acc1[8], acc2[16], db = 0.f;
#pragma unroll
  for (int q = 0; q < 8; q++) acc1[q] = 0.f;
#pragma unroll
  for (int q = 0; q < 16; q++) acc2[q] = 0.f;
  const int i1 = t >> 2, k1 = (t & 3) * 8;    // dW1 [i1][k1 + q]
  const int o2 = t >> 2, i2 = (t & 3) * 16;   // dW2 [o2][i2 + q]
  for (size_t rb = r0; rb < r1; rb += TR) {
    const int nr = (int)std::min<size_t>(TR, r1 - rb);
    for (int x = t; x < TR * FL_H; x += 256) {
      const int rr = x / FL_H, c = x % FL_H;
      const bool ok = rr < nr;
      sL1[rr][c] = ok ? L1[(rb + rr) * FL_H + c] : 0.f;
      sL2[rr][c] = ok ? L2[(rb + rr) * FL_H + c] : 0.f;
      sR2[rr][c] = ok ? R2[(rb + rr) * FL_H + c] : 0.f;
    }
    for (int x = t; x < TR * FL_E; x += 256) {
      const int rr = x / FL_E, c = x % FL_E;
      sR1[rr][c] = rr < nr ? R1[(rb + rr) * FL_E + c] : 0.f;
    }
    __syncthreads();
    for (int rr = 0; rr < nr; rr++) {
      const float l1 = sL1[rr][i1], l2 = sL2[rr][o2];
#pragma unroll
      for (int q = 0; q < 8; q++) acc1[q] += l1 * sR1[rr][k1 + q];
#pragma unroll
      for (int q = 0; q < 16; q++) acc2[q] += l2 * sR2[rr][i2 + q];
      if ((rb + rr) % P == 0) {  // potential-path rows give the bias gradients
        if (t < FL_H) db += sL1[rr][t];
        else if (t < 2 * FL_H) db += sL2[rr][t - FL_H];
      }
    }
    __syncthreads();
  }
  float *o = part + (size_t)blockIdx.x * NM;
#pragma unroll
  for (int q = 0; q < 8; q++) o[MO_W1 + i1 * FL_E + k1 + q] = acc1[q];
#pragma unroll
  for (int q = 0; q < 16; q++) o[MO_W2 + o2 * FL_H + i2 + q] = acc2[q];
  if (t < FL_H) o[MO_B1 + t] = db;
  else if (t < 2 * FL_H) o[MO_B2 + t - FL_H] = db;
  // output layer: dW3 [f][i] and db3 [f]
  for (int x = t; x < FL_NF * (FL_H + 1); x += 256) {
    const int f = x / (FL_H + 1), c = x % (FL_H + 1);
    float sum = 0.f;
    if (f < NF)
      for (int jj = jb; jj < je; jj++) sum += V3[((size_t)jj * NF + f) * (FL_H + 1) + c];
    if (c < FL_H) o[MO_W3 + f * FL_H + c] = sum;
    else o[MO_B3 + f] = sum;
  }
}

__global__ void sum_partials_kernel(const float *__restrict__ part, int nparts, float *out) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= NM) return;
  float s = 0.f;
  for (int c = 0; c < nparts; c++) s += part[(size_t)c * NM + o];
  out[o] = s;
}

__global__ void sum_loss_kernel(const float *__restrict__ l, int n, float *out) {
  __shared__ float sh[256];
  float s = 0.f;
  for (int i = threadIdx.x; i < n; i += 256) s += l[i];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0];
}

// ---- Adam -------------------------------------------------------------------
__global__ void adam_mlp_kernel(float *p, float *m, float *v, const float *g, int n, float lr, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = 0.9f * m[i] + 0.1f * gi, vi = 0.99f * v[i] + 0.01f * gi * gi;
  m[i] = mi; v[i] = vi;
  p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + 1e-15f);
}
__global__ void adam_table_kernel(float2 *p, float2 *m, float2 *v, unsigned long long *g, size_t n, float lr, float c1,
                                  float c2) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float ga = (float)((double)(long long)g[2 * i] * (1.0 / FIX_SCALE));
  const float gb = (float)((double)(long long)g[2 * i + 1] * (1.0 / FIX_SCALE));
  g[2 * i] = 0ull;
  g[2 * i + 1] = 0ull;
  float2 mi = m[i], vi = v[i], pi = p[i];
  mi.x = 0.9f * mi.x + 0.1f * ga; mi.y = 0.9f * mi.y + 0.1f * gb;
  vi.x = 0.99f * vi.x + 0.01f * ga * ga; vi.y = 0.99f * vi.y + 0.01f * gb * gb;
  pi.x -= lr * (mi.x * c1) / (sqrtf(vi.x * c2) + 1e-15f);
  pi.y -= lr * (mi.y * c1) / (sqrtf(vi.y * c2) + 1e-15f);
  m[i] = mi; v[i] = vi; p[i] = pi;
}

// ---- inference copies -------------------------------------------------------
struct FieldScales {
  float s[FL_NF];
};
__device__ __forceinline__ float bf16_rne(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }

__global__ void table_to_bf16_kernel(const float2 *__restrict__ t, size_t n, uint32_t *out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float2 v = t[i];
  out[i] = pack_bf16x2(v.x, v.y);
}

// FP32 inference copies and the tcgen05 B images from the master MLP (one CTA).
__global__ void pack_mlp_kernel(const float *__restrict__ m, int nf, FieldScales sc, float *inf, uint16_t *umma) {
  for (int t = threadIdx.x; t < FL_H * FL_E; t += blockDim.x) {
    const int i = t / FL_E, k = t % FL_E;
    const float w = bf16_rne(m[MO_W1 + t]);
    inf[FO_W1 + t] = w;
    inf[FO_W1T + k * FL_H + i] = w;
  }
  for (int t = threadIdx.x; t < FL_H * FL_H; t += blockDim.x) {
    const int o = t / FL_H, i = t % FL_H;
    const float w = bf16_rne(m[MO_W2 + t]);
    inf[FO_W2 + t] = w;
    inf[FO_W2T + i * FL_H + o] = w;
  }
  for (int t = threadIdx.x; t < FL_H; t += blockDim.x) {
    inf[FO_B1 + t] = m[MO_B1 + t];
    inf[FO_B2 + t] = m[MO_B2 + t];
  }
  for (int t = threadIdx.x; t < FL_NF * FL_H; t += blockDim.x) inf[FO_W3 + t] = (t / FL_H) < nf ? m[MO_W3 + t] : 0.f;
  if (threadIdx.x < FL_NF) {
    inf[FO_B3 + threadIdx.x] = (int)threadIdx.x < nf ? m[MO_B3 + threadIdx.x] : 0.f;
    inf[FO_S + threadIdx.x] = sc.s[threadIdx.x];
  }
  // B images, element (n, k) at (k / 8) * (N * 8) + n * 8 + (k % 8) (in bf16 units)
  auto put = [&](int base_bytes, int N, int n, int k, float v) {
    umma[base_bytes / 2 + (k / 8) * (N * 8) + n * 8 + (k % 8)] = __bfloat16_as_ushort(__float2bfloat16_rn(v));
  };
  for (int t = threadIdx.x; t < FL_H * FL_E; t += blockDim.x) {
    const int i = t / FL_E, j = t % FL_E;
    const float w = m[MO_W1 + t];
    put(FU_W1, FL_H, i, j, w);   // stage 1: B[n = i][k = j] = W1[i][j]
    put(FU_W1T, FL_E, j, i, w);  // stage 4: B[n = j][k = i] = W1[i][j]
  }
  for (int t = threadIdx.x; t < FL_H * FL_H; t += blockDim.x) {
    const int o = t / FL_H, i = t % FL_H;
    const float w = m[MO_W2 + t];
    put(FU_W2, FL_H, o, i, w);   // stage 2: B[n = o][k = i] = W2[o][i]
    put(FU_W2T, FL_H, i, o, w);  // stage 3: B[n = i][k = o] = W2[o][i]
  }
}

// ---- inference kernels (validation and ccs_field_eval) ----------------------
// Warp path: one warp per position; the site's fields (value and minus the
// gradient, 4 slots per position) as doubles.
__global__ void eval_warp_kernel(FieldK F, size_t n, const float4 *__restrict__ pos, int site, double *u,
                                 double *g, int8_t *exact) {
  const size_t w = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
  const int lane = threadIdx.x & 31;
  int fl[FL_SITE_FIELDS];
  const int nfo = site_fields(F, site, fl);
  for (size_t i = w; i < n; i += nw) {
    const float4 p = pos[i];
    const float x[3] = {p.x, p.y, p.z};
    float uu[FL_SITE_FIELDS], gg[FL_SITE_FIELDS][3];
    field_site_warp(F, x, nfo, fl, uu, gg);
    if (lane == 0) {
      for (int k = 0; k < nfo; k++) {
        u[4 * i + k] = uu[k];
        for (int a = 0; a < 3; a++) g[(4 * i + k) * 3 + a] = gg[k][a];
      }
      if (exact) exact[i] = field_exact(F, x[0], x[1], x[2]) ? 1 : 0;
    }
  }
}

// Tensor-core path: 128 positions per tile, CTAs stride over tiles.
__global__ void __launch_bounds__(TC_ROWS) eval_tc_kernel(FieldK F, size_t n, const float4 *__restrict__ pos,
                                                          int site, double *u, double *g, int8_t *exact,
                                                          int *error) {
  extern __shared__ __align__(1024) unsigned char dsm[];
  const uint32_t tmem = tc_setup(F, dsm);
  uint32_t phase = 0;
  int fl[FL_SITE_FIELDS];
  const int nfo = site_fields(F, site, fl);
  const size_t ntiles = (n + TC_ROWS - 1) / TC_ROWS;
  for (size_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const size_t i = tile * TC_ROWS + threadIdx.x;
    const bool use = i < n;
    float x[3] = {0.f, 0.f, 0.f};
    if (use) {
      const float4 p = pos[i];
      x[0] = p.x; x[1] = p.y; x[2] = p.z;
    }
    float e[FL_E], J[FL_E][3];
    field_encode(F, x, e, J);
    float uu[FL_SITE_FIELDS], gg[FL_SITE_FIELDS][3];
    if (!tc_site(F, dsm, tmem, phase, use, e, J, nfo, fl, uu, gg)) {
      if (threadIdx.x == 0) atomicExch(error, 2);
      break;
    }
    if (use) {
      for (int k = 0; k < nfo; k++) {
        u[4 * i + k] = uu[k];
        for (int a = 0; a < 3; a++) g[(4 * i + k) * 3 + a] = gg[k][a];
      }
      if (exact) exact[i] = field_exact(F, x[0], x[1], x[2]) ? 1 : 0;
    }
  }
  tc_teardown(tmem);
}

// Validation: warp inference of every field against the labels.  A sample's
// force error is the largest over the fields of |F - F*| in units of that
// field's RMS label gradient, its value error |u - u*| in units of the
// field's output scale; each coarse voxel keeps the largest force error of its
// samples (atomicMax on the float bits: errors are non-negative).
__global__ void validate_kernel(FieldK F, size_t n, const float4 *__restrict__ pos, const float *__restrict__ lab,
                                int nf, TrainGeo G, float evox_inv, int ev, float *err_f, float *err_u,
                                unsigned int *vox_err) {
  const size_t w = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
  const int lane = threadIdx.x & 31;
  for (size_t i = w; i < n; i += nw) {
    const float4 p = pos[i];
    const float x[3] = {p.x, p.y, p.z};
    float emax = 0.f, eu = 0.f;
    for (int f0i = 0; f0i < nf; f0i += FL_SITE_FIELDS) {
      int fl[FL_SITE_FIELDS];
      const int nfo = min(FL_SITE_FIELDS, nf - f0i);
      for (int k = 0; k < FL_SITE_FIELDS; k++) fl[k] = min(f0i + k, nf - 1);
      float uu[FL_SITE_FIELDS], ff[FL_SITE_FIELDS][3];
      field_site_warp(F, x, nfo, fl, uu, ff);
      for (int k = 0; k < nfo; k++) {
        const int fld = fl[k];
        const float *lb = lab + (i * nf + fld) * 4;
        const float dx = ff[k][0] - lb[1], dy = ff[k][1] - lb[2], dz = ff[k][2] - lb[3];
        emax = fmaxf(emax, sqrtf(dx * dx + dy * dy + dz * dz) / fmaxf(G.gs[fld], 1e-30f));
        eu = fmaxf(eu, fabsf(uu[k] - lb[0]) / fmaxf(G.s[fld], 1e-30f));
      }
    }
    if (lane == 0) {
      err_f[i] = emax;
      err_u[i] = eu;
      const int a = min(ev - 1, max(0, (int)floorf((x[0] - F.lo[0]) * evox_inv)));
      const int b = min(ev - 1, max(0, (int)floorf((x[1] - F.lo[1]) * evox_inv)));
      const int c = min(ev - 1, max(0, (int)floorf((x[2] - F.lo[2]) * evox_inv)));
      atomicMax(&vox_err[(size_t)a + (size_t)ev * ((size_t)b + (size_t)ev * (size_t)c)], __float_as_uint(emax));
    }
  }
}

// Fine voxels of every coarse voxel whose error exceeds the threshold.
__global__ void flag_err_voxels_kernel(FieldK F, const unsigned int *__restrict__ vox_err, int ev, int ratio,
                                       float thr, uint32_t *bits, unsigned long long *count) {
  const size_t cv = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (cv >= (size_t)ev * ev * ev) return;
  if (!(__uint_as_float(vox_err[cv]) > thr)) return;
  atomicAdd(count, 1ull);
  const int a = (int)(cv % ev), b = (int)((cv / ev) % ev), c = (int)(cv / ((size_t)ev * ev));
  for (int k = c * ratio; k < min(F.vz, (c + 1) * ratio); k++)
    for (int j = b * ratio; j < min(F.vy, (b + 1) * ratio); j++)
      for (int i = a * ratio; i < min(F.vx, (a + 1) * ratio); i++) {
        const uint32_t v = (uint32_t)i + (uint32_t)F.vx * ((uint32_t)j + (uint32_t)F.vy * (uint32_t)k);
        atomicOr(&bits[v >> 5], 1u << (v & 31u));
      }
}

__global__ void popcount_kernel(const uint32_t *__restrict__ bits, size_t nwords, unsigned long long *count) {
  unsigned long long c = 0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nwords; i += (size_t)gridDim.x * blockDim.x)
    c += __popc(bits[i]);
  atomicAdd(count, c);
}

// ---- host helpers -----------------------------------------------------------
double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

template <typename P> int dalloc(ccs_ctx *c, P *&p, size_t bytes) {
  dfree(p);
  if (cudaMalloc((void **)&p, bytes) != cudaSuccess) {
    cudaGetLastError();
    p = nullptr;
    return fail(c, CCS_ERR_NOMEM, "cudaMalloc of %zu bytes for the learned field", bytes);
  }
  return CCS_OK;
}

void free_state(FieldState *fs) {
  dfree(fs->table); dfree(fs->tm); dfree(fs->tv); dfree(fs->tgrad);
  dfree(fs->mlp); dfree(fs->mm); dfree(fs->mv); dfree(fs->mgrad);
  dfree(fs->table_bf16); dfree(fs->mlp_inf); dfree(fs->umma); dfree(fs->bits);
  dfree(fs->spos); dfree(fs->slab);
  dfree(fs->L1); dfree(fs->R1); dfree(fs->L2); dfree(fs->R2); dfree(fs->V3); dfree(fs->part); dfree(fs->lossbuf);
  dfree(fs->bidx);
}

// The geometry and per-field scales and floors the training kernel reads.
void refresh_geo(FieldState *fs) {
  for (int f = 0; f < FL_NF; f++) {
    fs->geo.s[f] = (float)fs->s[f];
    fs->geo.gs[f] = (float)fs->gs[f];
    fs->geo.u0[f] = (float)(fs->p.u0 * fs->s[f]);
    fs->geo.f0[f] = (float)(fs->p.f0 * fs->gs[f]);
  }
}

// The fields of a context: the far potential of each gas site type (with
// its LJ parameter set and charge), then, with the induced dipole, the three
// far-field components; the field of each site and the dipole's site.
void field_layout(const ccs_ctx *c, FieldState *fs) {
  FieldKind &k = fs->kinds;
  std::memset(&k, 0, sizeof k);
  const int gas = c->p.gas;
  const bool coul = c->coul_on != 0;
  int nf = 0;
  if (gas == CCS_GAS_N2) {  // N, N, central charge (GasBuffer.cpp:79-115)
    k.lj[0] = 1; k.q[0] = coul ? -0.4825 : 0.0;
    k.lj[1] = 0; k.q[1] = coul ? 0.965 : 0.0;
    nf = 2;
    fs->site_field[0] = fs->site_field[1] = 0; fs->site_field[2] = 1;
    fs->dip_site = c->dip_on ? 2 : -1;
  } else if (gas == CCS_GAS_CO2) {  // O, C, O (GasBuffer.cpp:116-165)
    k.lj[0] = 1; k.q[0] = coul ? -0.3256 : 0.0;
    k.lj[1] = 2; k.q[1] = coul ? 0.6512 : 0.0;
    nf = 2;
    fs->site_field[0] = fs->site_field[2] = 0; fs->site_field[1] = 1;
    fs->dip_site = c->dip_on ? 1 : -1;
  } else {  // atoms: LJ only (neutral probe)
    k.lj[0] = 1; k.q[0] = 0.0;
    nf = 1;
    fs->site_field[0] = fs->site_field[1] = fs->site_field[2] = 0;
    fs->dip_site = c->dip_on ? 0 : -1;
  }
  fs->efield = nf;
  if (fs->dip_site >= 0)
    for (int a = 0; a < 3; a++) { k.kind[nf] = 1; k.comp[nf] = a; nf++; }
  fs->nf = nf;
}

// Geometry (domain cube, grids, bitmap dimensions), parameter memory and
// random initial parameters.
int setup_geometry(ccs_ctx *c, FieldState *fs, const ccs_field_params &p) {
  fs->p = p;
  field_layout(c, fs);
  // the region a site can reach while the probe is within the force reach of
  // the target's bounding box, plus a margin
  const double margin = c->reach + 2.5 + 1.0;
  double side = 0.0, cen[3];
  for (int d = 0; d < 3; d++) {
    side = std::max(side, c->bb_hi[d] - c->bb_lo[d] + 2.0 * margin);
    cen[d] = 0.5 * (c->bb_lo[d] + c->bb_hi[d]);
  }
  fs->side = side;
  FieldK &K = fs->k;
  std::memset(&K, 0, sizeof K);
  for (int d = 0; d < 3; d++) {
    fs->lo[d] = cen[d] - 0.5 * side;
    K.lo[d] = (float)fs->lo[d];
    fs->geo.lo[d] = K.lo[d];
  }
  K.side = (float)side;
  const double growth = std::exp((std::log((double)p.finest_res) - std::log((double)p.base_res)) / (FL_LEVELS - 1));
  fs->rows = (size_t)1 << p.log2_table;
  for (int l = 0; l < FL_LEVELS; l++) {
    const int r = (int)std::floor(p.base_res * std::pow(growth, l) + 1e-9);
    K.res[l] = r;
    const double r1 = (double)r + 1.0;
    K.dense[l] = r1 * r1 * r1 <= (double)fs->rows ? 1 : 0;
    K.scale[l] = (float)(r / side);
    fs->geo.res[l] = r;
    fs->geo.dense[l] = K.dense[l];
    fs->geo.scale[l] = K.scale[l];
  }
  K.tmask = (uint32_t)(fs->rows - 1);
  K.log2t = p.log2_table;
  fs->geo.tmask = K.tmask;
  fs->geo.log2t = K.log2t;
  const int nv = (int)std::ceil(side / p.voxel);
  K.vx = K.vy = K.vz = nv;
  K.vox_inv = (float)(1.0 / p.voxel);
  K.nf = fs->nf;
  for (int s = 0; s < 3; s++) K.site_field[s] = fs->site_field[s];
  K.dip_site = fs->dip_site;
  K.efield = fs->efield;
  K.r_in = (float)p.r_in;
  K.r_out = (float)p.r_out;
  fs->nwords = ((size_t)nv * nv * nv + 31) / 32;
  const size_t nt = (size_t)FL_LEVELS * fs->rows;
  int rc;
  if ((rc = dalloc(c, fs->table, nt * sizeof(float2))) || (rc = dalloc(c, fs->tm, nt * sizeof(float2))) ||
      (rc = dalloc(c, fs->tv, nt * sizeof(float2))) || (rc = dalloc(c, fs->tgrad, nt * 2 * sizeof(unsigned long long))) ||
      (rc = dalloc(c, fs->mlp, NM * sizeof(float))) || (rc = dalloc(c, fs->mm, NM * sizeof(float))) ||
      (rc = dalloc(c, fs->mv, NM * sizeof(float))) || (rc = dalloc(c, fs->mgrad, NM * sizeof(float))) ||
      (rc = dalloc(c, fs->table_bf16, nt * sizeof(uint32_t))) || (rc = dalloc(c, fs->mlp_inf, FO_TOTAL * sizeof(float))) ||
      (rc = dalloc(c, fs->umma, FU_BYTES)) || (rc = dalloc(c, fs->bits, fs->nwords * sizeof(uint32_t))))
    return rc;
  K.table = fs->table_bf16;
  K.exact_bits = fs->bits;
  K.mlp = fs->mlp_inf;
  K.umma = fs->umma;
  // initial parameters: table uniform in +-1e-4, He/Kaiming-normal weights, zero biases
  std::vector<float2> t0(nt);
  uint64_t st = mix64(p.seed ^ 0x7ab1e);
  for (size_t i = 0; i < nt; i++) {
    const uint64_t a = mix64(st + 2 * i), b = mix64(st + 2 * i + 1);
    t0[i] = make_float2((float)((double)(a >> 11) * (1.0 / 9007199254740992.0) * 2e-4 - 1e-4),
                        (float)((double)(b >> 11) * (1.0 / 9007199254740992.0) * 2e-4 - 1e-4));
  }
  std::vector<float> m0(NM, 0.f);
  uint64_t sm = mix64(p.seed ^ 0x31f);
  auto normal = [&]() {  // Box-Muller from two hashed uniforms
    const double u1 = ((double)(mix64(sm++) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    const double u2 = (double)(mix64(sm++) >> 11) * (1.0 / 9007199254740992.0);
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  };
  for (int i = 0; i < FL_H * FL_E; i++) m0[MO_W1 + i] = (float)(normal() * std::sqrt(2.0 / FL_E));
  for (int i = 0; i < FL_H * FL_H; i++) m0[MO_W2 + i] = (float)(normal() * std::sqrt(2.0 / FL_H));
  for (int i = 0; i < FL_NF * FL_H; i++) m0[MO_W3 + i] = (float)(normal() * std::sqrt(1.0 / FL_H));
  CK(to_dev(c, fs->table, t0.data(), nt * sizeof(float2)));
  CK(to_dev(c, fs->mlp, m0.data(), NM * sizeof(float)));
  CK(zero_dev(c, fs->tm, nt * sizeof(float2)));
  CK(zero_dev(c, fs->tv, nt * sizeof(float2)));
  CK(zero_dev(c, fs->tgrad, nt * 2 * sizeof(unsigned long long)));
  CK(zero_dev(c, fs->mm, NM * sizeof(float)));
  CK(zero_dev(c, fs->mv, NM * sizeof(float)));
  // exact-evaluation bitmap: voxels whose centre is within fallback_radius +
  // half a voxel diagonal of an atom (every point within fallback_radius of an
  // atom then lies in a flagged voxel)
  CK(zero_dev(c, fs->bits, fs->nwords * sizeof(uint32_t)));
  const float R = (float)(p.fallback_radius + 0.5 * std::sqrt(3.0) * p.voxel);
  bitmap_atoms_kernel<<<(c->natoms + 127) / 128, 128, 0, c->stream>>>(c->d_xyzq32, c->natoms, K, (float)p.voxel, R,
                                                                     fs->bits);
  CK(cudaGetLastError());
  for (int f = 0; f < FL_NF; f++) fs->s[f] = fs->gs[f] = 1.0;
  refresh_geo(fs);
  return CCS_OK;
}

int pack_inference(ccs_ctx *c, FieldState *fs) {
  const size_t nt = (size_t)FL_LEVELS * fs->rows;
  table_to_bf16_kernel<<<(unsigned)((nt + 255) / 256), 256, 0, c->stream>>>(fs->table, nt, fs->table_bf16);
  CK(cudaGetLastError());
  FieldScales sc;
  for (int f = 0; f < FL_NF; f++) sc.s[f] = (float)fs->s[f];
  pack_mlp_kernel<<<1, 256, 0, c->stream>>>(fs->mlp, fs->nf, sc, fs->mlp_inf, reinterpret_cast<uint16_t *>(fs->umma));
  CK(cudaGetLastError());
  refresh_geo(fs);
  return CCS_OK;
}

// n samples drawn with the given seed stream into (pos, labels)
int draw_samples(ccs_ctx *c, FieldState *fs, size_t n, uint64_t seed, float4 *&pos, float *&lab, double *ms_sample,
                 double *ms_label) {
  const ccs_field_params &p = fs->p;
  cudaStream_t s = c->stream;
  double t0 = now_ms();
  int rc = dalloc(c, pos, n * sizeof(float4));
  if (rc) return rc;
  // candidates in chunks until n are kept (stable compaction: deterministic order)
  size_t have = 0;
  uint64_t first = 0;
  const size_t chunk = std::max<size_t>(1 << 20, std::min<size_t>(n, 1 << 24));
  float4 *cand = nullptr, *stage = nullptr;
  char *keep = nullptr;
  size_t *d_num = nullptr;
  void *tmp = nullptr;
  size_t tmp_bytes = 0;
  auto cleanup = [&]() { dfree(cand); dfree(stage); dfree(keep); dfree(d_num); dfree(tmp); };
  if ((rc = dalloc(c, cand, chunk * sizeof(float4))) || (rc = dalloc(c, stage, chunk * sizeof(float4))) ||
      (rc = dalloc(c, keep, chunk)) || (rc = dalloc(c, d_num, sizeof(size_t)))) {
    cleanup();
    return rc;
  }
  if (cub::DeviceSelect::Flagged(nullptr, tmp_bytes, cand, keep, stage, d_num, (int)chunk) != cudaSuccess ||
      (rc = dalloc(c, tmp, tmp_bytes))) {
    cleanup();
    return rc ? rc : fail(c, CCS_ERR_CUDA, "sample compaction");
  }
  for (int rounds = 0; have < n && rounds < 256; rounds++) {
    sample_kernel<<<(unsigned)((chunk + 255) / 256), 256, 0, s>>>(
        seed, first, chunk, c->d_xyzq32, c->natoms, fs->k, (float)p.near_fraction, (float)p.fallback_radius,
        (float)p.near_shell, cand, keep);
    first += chunk;
    size_t got = 0, tb = tmp_bytes;
    if (cub::DeviceSelect::Flagged(tmp, tb, cand, keep, stage, d_num, (int)chunk, s) != cudaSuccess ||
        cudaMemcpyAsync(&got, d_num, sizeof(size_t), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
      rc = fail(c, CCS_ERR_CUDA, "sampling: %s", cudaGetErrorString(cudaGetLastError()));
      break;
    }
    const size_t take = std::min(got, n - have);
    if (cudaMemcpyAsync(pos + have, stage, take * sizeof(float4), cudaMemcpyDeviceToDevice, s) != cudaSuccess) {
      rc = fail(c, CCS_ERR_CUDA, "sample copy");
      break;
    }
    have += take;
  }
  cleanup();
  if (rc) return rc;
  if (have < n) return fail(c, CCS_ERR_INVALID, "learned field: only %zu of %zu samples found outside the exact zone", have, n);
  CK(cudaStreamSynchronize(s));
  double t1 = now_ms();
  if (ms_sample) *ms_sample += t1 - t0;
  // labels: the far parts of every field at every sample
  if ((rc = dalloc(c, lab, n * fs->nf * 4 * sizeof(float)))) return rc;
  KParams kp = base_params(c);
  kp.field = fs->k;
  far_label_kernel<<<(unsigned)std::min<size_t>((n + 7) / 8, (size_t)c->sm_count * 64), 256, 0, s>>>(
      kp, fs->kinds, fs->nf, n, pos, lab);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(s));
  if (ms_label) *ms_label += now_ms() - t1;
  return rc;
}

int ensure_scratch(ccs_ctx *c, FieldState *fs, size_t B) {
  if (B <= fs->scratch_batch) return CCS_OK;
  const int P = 1 + fs->nf;
  const size_t nparts = (B + WG_CH - 1) / WG_CH;
  int rc;
  if ((rc = dalloc(c, fs->L1, B * P * FL_H * sizeof(float))) || (rc = dalloc(c, fs->R1, B * P * FL_E * sizeof(float))) ||
      (rc = dalloc(c, fs->L2, B * P * FL_H * sizeof(float))) || (rc = dalloc(c, fs->R2, B * P * FL_H * sizeof(float))) ||
      (rc = dalloc(c, fs->V3, B * fs->nf * (FL_H + 1) * sizeof(float))) ||
      (rc = dalloc(c, fs->part, nparts * NM * sizeof(float))) || (rc = dalloc(c, fs->lossbuf, B * sizeof(float))) ||
      (rc = dalloc(c, fs->bidx, B * sizeof(int))))
    return rc;
  fs->scratch_batch = B;
  fs->part_rows = nparts;
  return CCS_OK;
}

constexpr size_t TRAIN_SMEM = (size_t)(2 * FL_H * FL_E + 2 * FL_H * FL_H + 2 * FL_H + FL_NF * FL_H + FL_NF) * sizeof(float);

// The per-sample pass (forward, backward, table gradients) and the per-chunk
// weight-gradient partial sums of one batch, for NF fields.
template <int NF>
void launch_train(ccs_ctx *c, FieldState *fs, const float4 *pos, const float *lab, int B, int grid, float invB,
                  cudaStream_t s) {
  train_kernel<NF><<<grid, 256, TRAIN_SMEM, s>>>(fs->table, fs->mlp, fs->geo, pos, lab, fs->bidx, B,
                                                 (float)fs->p.lam_u, invB, fs->L1, fs->R1, fs->L2, fs->R2, fs->V3,
                                                 fs->lossbuf, fs->tgrad);
  const int nparts = (B + WG_CH - 1) / WG_CH;
  wgrad_kernel<NF><<<nparts, 256, 0, s>>>(fs->L1, fs->R1, fs->L2, fs->R2, fs->V3, B, fs->part);
}

// Loss gradients of one batch (indices already in fs->bidx) into fs->mgrad
// and fs->tgrad; the batch's mean loss into *loss_dev.
int grad_step(ccs_ctx *c, FieldState *fs, const float4 *pos, const float *lab, int B, float *loss_dev) {
  cudaStream_t s = c->stream;
  const int grid = std::max(1, std::min(c->sm_count * 8, (B + 7) / 8));
  const float invB = 1.0f / (float)B;
  switch (fs->nf) {
    case 1: launch_train<1>(c, fs, pos, lab, B, grid, invB, s); break;
    case 2: launch_train<2>(c, fs, pos, lab, B, grid, invB, s); break;
    case 4: launch_train<4>(c, fs, pos, lab, B, grid, invB, s); break;
    default: launch_train<5>(c, fs, pos, lab, B, grid, invB, s); break;
  }
  CK(cudaGetLastError());
  const int nparts = (B + WG_CH - 1) / WG_CH;
  sum_partials_kernel<<<(NM + 255) / 256, 256, 0, s>>>(fs->part, nparts, fs->mgrad);
  CK(cudaGetLastError());
  if (loss_dev) {
    sum_loss_kernel<<<1, 256, 0, s>>>(fs->lossbuf, B, loss_dev);
    CK(cudaGetLastError());
  }
  return CCS_OK;
}

int attr_once(ccs_ctx *c) {
  static bool done[64] = {};  // per device: the kernels' dynamic shared memory limits
  if (c->device < 0 || c->device >= 64) return fail(c, CCS_ERR_INVALID, "device number");
  if (done[c->device]) return CCS_OK;
  CK(cudaFuncSetAttribute(train_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TRAIN_SMEM));
  CK(cudaFuncSetAttribute(train_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TRAIN_SMEM));
  CK(cudaFuncSetAttribute(train_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TRAIN_SMEM));
  CK(cudaFuncSetAttribute(train_kernel<5>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TRAIN_SMEM));
  CK(cudaFuncSetAttribute(eval_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM_BYTES));
  done[c->device] = true;
  return CCS_OK;
}

int check_ctx(ccs_ctx *c) {
  if (!c) return CCS_ERR_INVALID;
  if (!c->have_target) return fail(c, CCS_ERR_INVALID, "no target set");
  if (c->p.precision != CCS_PREC_FP32) return fail(c, CCS_ERR_UNSUPPORTED, "the learned field needs FP32 precision");
  if (c->allpairs) return fail(c, CCS_ERR_UNSUPPORTED, "the learned field needs cutoffs (force types 2, 4 or 6)");
  if (cudaSetDevice(c->device) != cudaSuccess) return fail(c, CCS_ERR_CUDA, "cudaSetDevice");
  return attr_once(c);
}

int check_params(ccs_ctx *c, const ccs_field_params *p) {
  if (!p) return fail(c, CCS_ERR_INVALID, "field parameters are required");
  if (p->log2_table < 10 || p->log2_table > 22) return fail(c, CCS_ERR_INVALID, "log2_table must be 10..22");
  if (p->base_res < 2 || p->finest_res < p->base_res || p->finest_res > 1 << 16)
    return fail(c, CCS_ERR_INVALID, "need 2 <= base_res <= finest_res <= 65536");
  if (!(p->fallback_radius > 0) || !(p->voxel > 0) || !(p->err_voxel >= p->voxel))
    return fail(c, CCS_ERR_INVALID, "fallback_radius, voxel > 0 and err_voxel >= voxel are required");
  if (p->samples < 1024 || p->batch < 32 || p->iterations < 0 || p->validation < 0)
    return fail(c, CCS_ERR_INVALID, "samples >= 1024, batch >= 32, iterations and validation >= 0");
  if ((size_t)p->batch > (size_t)p->samples) return fail(c, CCS_ERR_INVALID, "batch exceeds samples");
  if (!(p->r_in > 0) || !(p->r_out > p->r_in)) return fail(c, CCS_ERR_INVALID, "need 0 < r_in < r_out");
  return CCS_OK;
}

void fill_report(const FieldState *fs, ccs_field_report *r) {
  if (!r) return;
  for (int d = 0; d < 3; d++) r->domain_lo[d] = fs->lo[d];
  r->domain_side = fs->side;
  r->levels = FL_LEVELS;
  r->dense_levels = 0;
  for (int l = 0; l < FL_LEVELS; l++) {
    r->res[l] = fs->k.res[l];
    r->dense_levels += fs->k.dense[l];
  }
  r->nfields = fs->nf;
  r->log2_table = fs->p.log2_table;
  for (int f = 0; f < FL_NF; f++) {
    r->output_scale[f] = fs->s[f];
    r->gradient_scale[f] = fs->gs[f];
  }
}

}  // namespace

void ccs_internal::field_kparams(const ccs_ctx *c, KParams &k) {
  if (c->field_on && c->field && c->field->ready) {
    k.field = c->field->k;
    k.field.on = 1;
  } else {
    std::memset(&k.field, 0, sizeof k.field);
  }
}

void ccs_internal::field_free(ccs_ctx *c) {
  if (!c->field) return;
  free_state(c->field);
  delete c->field;
  c->field = nullptr;
  c->field_on = false;
}

extern "C" {

void ccs_field_params_default(ccs_field_params *p) {
  if (!p) return;
  std::memset(p, 0, sizeof *p);
  p->samples = 4000000;
  p->iterations = 6000;
  p->batch = 32768;
  p->log2_table = 20;
  p->base_res = 8;
  p->finest_res = 128;
  p->validation = 1 << 20;
  p->fallback_radius = 2.0;
  p->voxel = 0.5;
  p->err_voxel = 2.0;
  p->err_threshold = 0.0;
  p->near_fraction = 0.5;
  p->near_shell = 6.0;
  p->lr = 1e-2;
  p->lam_u = 0.1;
  p->u0 = 0.05;
  p->f0 = 0.05;
  p->seed = 2104;
  p->r_in = 6.0;
  p->r_out = 12.0;
}

int ccs_field_setup(ccs_ctx *c, const ccs_field_params *p, ccs_field_report *report) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if ((rc = check_params(c, p))) return rc;
  field_free(c);
  c->field = new (std::nothrow) FieldState();
  if (!c->field) return fail(c, CCS_ERR_NOMEM, "learned field state");
  FieldState *fs = c->field;
  if ((rc = setup_geometry(c, fs, *p)) || (rc = pack_inference(c, fs))) {
    field_free(c);
    return rc;
  }
  CK(cudaStreamSynchronize(c->stream));
  fs->ready = true;
  if (report) {
    std::memset(report, 0, sizeof *report);
    fill_report(fs, report);
  }
  return CCS_OK;
}

int ccs_field_train(ccs_ctx *c, const ccs_field_params *p, ccs_field_report *report) {
  int rc = ccs_field_setup(c, p, nullptr);
  if (rc) return rc;
  FieldState *fs = c->field;
  fs->ready = false;
  cudaStream_t s = c->stream;
  ccs_field_report rep;
  std::memset(&rep, 0, sizeof rep);
  auto bail = [&](int code) {
    field_free(c);
    return code;
  };
  // ---- samples and labels
  fs->nsamples = (size_t)p->samples;
  if ((rc = draw_samples(c, fs, fs->nsamples, p->seed, fs->spos, fs->slab, &rep.sample_ms, &rep.label_ms)))
    return bail(rc);
  rep.samples = (int64_t)fs->nsamples;
  {  // per field: output scale = RMS of its values, gradient scale = RMS of |gradient|
    std::vector<float> lab(fs->nsamples * fs->nf * 4);
    if (to_host(c, lab.data(), fs->slab, lab.size() * sizeof(float)) != cudaSuccess)
      return bail(fail(c, CCS_ERR_CUDA, "label copy"));
    for (int f = 0; f < fs->nf; f++) {
      double su = 0.0, sg = 0.0;
      for (size_t i = 0; i < fs->nsamples; i++) {
        const float *l = &lab[(i * fs->nf + f) * 4];
        su += (double)l[0] * l[0];
        sg += (double)l[1] * l[1] + (double)l[2] * l[2] + (double)l[3] * l[3];
      }
      fs->s[f] = std::max(1e-12, std::sqrt(su / (double)fs->nsamples));
      fs->gs[f] = std::max(1e-12, std::sqrt(sg / (double)fs->nsamples));
      rep.output_scale[f] = fs->s[f];
      rep.gradient_scale[f] = fs->gs[f];
    }
    refresh_geo(fs);
  }
  // ---- training
  const int B = p->batch;
  if ((rc = ensure_scratch(c, fs, (size_t)B))) return bail(rc);
  float *d_loss = nullptr;
  if ((rc = dalloc(c, d_loss, 2 * sizeof(float)))) return bail(rc);
  const double t0 = now_ms();
  const size_t nt = (size_t)FL_LEVELS * fs->rows;
  for (int it = 0; it < p->iterations; it++) {
    batch_kernel<<<(B + 255) / 256, 256, 0, s>>>(p->seed, (uint64_t)it, B, fs->nsamples, fs->bidx);
    const bool rec = it == 0 || it == p->iterations - 1;
    rc = grad_step(c, fs, fs->spos, fs->slab, B, rec ? d_loss + (it == 0 ? 0 : 1) : nullptr);
    if (rc) break;
    const double t = it + 1;
    const float lr = (float)(p->lr * std::pow(0.1, (double)it / std::max(1, p->iterations)));
    const float c1 = (float)(1.0 / (1.0 - std::pow(0.9, t))), c2 = (float)(1.0 / (1.0 - std::pow(0.99, t)));
    adam_mlp_kernel<<<(NM + 255) / 256, 256, 0, s>>>(fs->mlp, fs->mm, fs->mv, fs->mgrad, NM, lr, c1, c2);
    adam_table_kernel<<<(unsigned)((nt + 255) / 256), 256, 0, s>>>(fs->table, fs->tm, fs->tv, fs->tgrad, nt, lr, c1, c2);
    if (cudaGetLastError() != cudaSuccess) { rc = fail(c, CCS_ERR_CUDA, "training step launch"); break; }
  }
  if (!rc && cudaStreamSynchronize(s) != cudaSuccess) rc = fail(c, CCS_ERR_CUDA, "training");
  if (rc) { dfree(d_loss); return bail(rc); }
  rep.train_ms = now_ms() - t0;
  float hl[2] = {0.f, 0.f};
  to_host(c, hl, d_loss, sizeof hl);
  dfree(d_loss);
  rep.first_loss = hl[0];
  rep.final_loss = p->iterations > 1 ? hl[1] : hl[0];
  if ((rc = pack_inference(c, fs))) return bail(rc);
  // training samples are no longer needed
  dfree(fs->spos); dfree(fs->slab);
  dfree(fs->L1); dfree(fs->R1); dfree(fs->L2); dfree(fs->R2); dfree(fs->V3); dfree(fs->part); dfree(fs->lossbuf);
  dfree(fs->bidx);
  fs->scratch_batch = 0;
  // ---- validation on fresh samples: error statistics and error voxels
  if (p->validation > 0) {
    const double tv0 = now_ms();
    float4 *vpos = nullptr;
    float *vlab = nullptr;
    const size_t nv = (size_t)p->validation;
    if ((rc = draw_samples(c, fs, nv, p->seed ^ 0x5eedf00dull, vpos, vlab, nullptr, nullptr))) return bail(rc);
    const int ev = (int)std::ceil(fs->side / p->err_voxel);
    const int ratio = std::max(1, (int)std::lround(p->err_voxel / p->voxel));
    float *ef = nullptr, *eu = nullptr;
    unsigned int *verr = nullptr;
    unsigned long long *cnt = nullptr;
    if ((rc = dalloc(c, ef, nv * sizeof(float))) || (rc = dalloc(c, eu, nv * sizeof(float))) ||
        (rc = dalloc(c, verr, (size_t)ev * ev * ev * sizeof(unsigned int))) ||
        (rc = dalloc(c, cnt, 2 * sizeof(unsigned long long)))) {
      dfree(vpos); dfree(vlab); dfree(ef); dfree(eu); dfree(verr); dfree(cnt);
      return bail(rc);
    }
    cudaMemsetAsync(verr, 0, (size_t)ev * ev * ev * sizeof(unsigned int), s);
    cudaMemsetAsync(cnt, 0, 2 * sizeof(unsigned long long), s);
    FieldK K = fs->k;
    validate_kernel<<<c->sm_count * 8, 256, 0, s>>>(K, nv, vpos, vlab, fs->nf, fs->geo,
                                                     (float)(1.0 / p->err_voxel), ev, ef, eu, verr);
    if (p->err_threshold > 0)  // error voxels switch to exact evaluation (0: none)
      flag_err_voxels_kernel<<<(unsigned)(((size_t)ev * ev * ev + 255) / 256), 256, 0, s>>>(
          K, verr, ev, ratio, (float)p->err_threshold, fs->bits, cnt);
    popcount_kernel<<<c->sm_count * 4, 256, 0, s>>>(fs->bits, fs->nwords, cnt + 1);
    std::vector<float> hf(nv), hu(nv);
    unsigned long long hc[2] = {0, 0};
    const bool ok = cudaGetLastError() == cudaSuccess && cudaStreamSynchronize(s) == cudaSuccess &&
                    to_host(c, hf.data(), ef, nv * sizeof(float)) == cudaSuccess &&
                    to_host(c, hu.data(), eu, nv * sizeof(float)) == cudaSuccess &&
                    to_host(c, hc, cnt, sizeof hc) == cudaSuccess;
    dfree(vpos); dfree(vlab); dfree(ef); dfree(eu); dfree(verr); dfree(cnt);
    if (!ok) return bail(fail(c, CCS_ERR_CUDA, "validation"));
    double sf = 0.0, su = 0.0;
    for (size_t i = 0; i < nv; i++) { sf += (double)hf[i] * hf[i]; su += (double)hu[i] * hu[i]; }
    std::vector<float> sorted(hf);
    const size_t q = std::min(nv - 1, (size_t)(0.99 * (double)nv));
    std::nth_element(sorted.begin(), sorted.begin() + q, sorted.end());
    rep.val_force_rel_rms = std::sqrt(sf / (double)nv);
    rep.val_force_rel_p99 = sorted[q];
    rep.val_u_rel_rms = std::sqrt(su / (double)nv);
    rep.err_voxels = (int64_t)hc[0];
    rep.exact_fraction = (double)hc[1] / ((double)fs->k.vx * fs->k.vy * fs->k.vz);
    rep.validate_ms = now_ms() - tv0;
  } else {
    unsigned long long *cnt = nullptr;
    if ((rc = dalloc(c, cnt, sizeof(unsigned long long)))) return bail(rc);
    cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), s);
    popcount_kernel<<<c->sm_count * 4, 256, 0, s>>>(fs->bits, fs->nwords, cnt);
    unsigned long long hc = 0;
    to_host(c, &hc, cnt, sizeof hc);
    dfree(cnt);
    rep.exact_fraction = (double)hc / ((double)fs->k.vx * fs->k.vy * fs->k.vz);
  }
  fill_report(fs, &rep);
  fs->ready = true;
  if (report) *report = rep;
  return CCS_OK;
}

int ccs_field_enable(ccs_ctx *c, int on) {
  if (!c) return CCS_ERR_INVALID;
  if (on && !(c->field && c->field->ready)) return fail(c, CCS_ERR_INVALID, "no learned field: call ccs_field_train");
  c->field_on = on != 0;
  return CCS_OK;
}

int ccs_field_eval(ccs_ctx *c, size_t n, int site, const double *pos, int path, double *u, double *g,
                   int8_t *exact, int32_t *nfields) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!(c->field && c->field->ready)) return fail(c, CCS_ERR_INVALID, "no learned field");
  FieldState *fs = c->field;
  const int ns = is_molecule(c->p.gas) ? 3 : 1;
  if (site < 0 || site >= ns) return fail(c, CCS_ERR_INVALID, "site out of range");
  if (path != 0 && path != 1) return fail(c, CCS_ERR_INVALID, "path must be 0 (tensor cores) or 1 (warp)");
  if (nfields) *nfields = site == fs->dip_site ? 4 : 1;
  if (n == 0) return CCS_OK;
  if (!pos || !u || !g) return fail(c, CCS_ERR_INVALID, "pos, u and g are required");
  std::vector<float4> hp(n);
  for (size_t i = 0; i < n; i++) hp[i] = make_float4((float)pos[3 * i], (float)pos[3 * i + 1], (float)pos[3 * i + 2], 0.f);
  float4 *dp = nullptr;
  double *du = nullptr, *dg = nullptr;
  int8_t *dx = nullptr;
  int *derr = nullptr;
  auto cleanup = [&]() { dfree(dp); dfree(du); dfree(dg); dfree(dx); dfree(derr); };
  if ((rc = dalloc(c, dp, n * sizeof(float4))) || (rc = dalloc(c, du, n * 4 * sizeof(double))) ||
      (rc = dalloc(c, dg, n * 12 * sizeof(double))) || (rc = dalloc(c, dx, n)) || (rc = dalloc(c, derr, sizeof(int)))) {
    cleanup();
    return rc;
  }
  int herr = 0;
  bool ok = to_dev(c, dp, hp.data(), n * sizeof(float4)) == cudaSuccess &&
            zero_dev(c, du, n * 4 * sizeof(double)) == cudaSuccess &&
            zero_dev(c, dg, n * 12 * sizeof(double)) == cudaSuccess &&
            zero_dev(c, derr, sizeof(int)) == cudaSuccess;
  if (ok) {
    if (path == 0) {
      const size_t tiles = (n + TC_ROWS - 1) / TC_ROWS;
      const unsigned grid = (unsigned)std::min<size_t>(tiles, (size_t)c->sm_count * 2);
      eval_tc_kernel<<<grid, TC_ROWS, TC_SMEM_BYTES, c->stream>>>(fs->k, n, dp, site, du, dg, dx, derr);
    } else {
      eval_warp_kernel<<<(unsigned)std::min<size_t>((n + 7) / 8, (size_t)c->sm_count * 16), 256, 0, c->stream>>>(
          fs->k, n, dp, site, du, dg, dx);
    }
    ok = cudaGetLastError() == cudaSuccess && cudaStreamSynchronize(c->stream) == cudaSuccess &&
         to_host(c, u, du, n * 4 * sizeof(double)) == cudaSuccess &&
         to_host(c, g, dg, n * 12 * sizeof(double)) == cudaSuccess &&
         (!exact || to_host(c, exact, dx, n) == cudaSuccess) &&
         to_host(c, &herr, derr, sizeof(int)) == cudaSuccess;
  }
  cleanup();
  if (!ok) return fail(c, CCS_ERR_CUDA, "field evaluation: %s", cudaGetErrorString(cudaGetLastError()));
  if (herr) return fail(c, CCS_ERR_TIMEOUT, "field evaluation: a tensor-core stage did not complete");
  return CCS_OK;
}

int ccs_field_labels(ccs_ctx *c, size_t n, const double *pos, double *labels) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!c->field) return fail(c, CCS_ERR_INVALID, "no learned field: call ccs_field_setup");
  if (n == 0) return CCS_OK;
  if (!pos || !labels) return fail(c, CCS_ERR_INVALID, "pos and labels are required");
  FieldState *fs = c->field;
  std::vector<float4> hp(n);
  for (size_t i = 0; i < n; i++) hp[i] = make_float4((float)pos[3 * i], (float)pos[3 * i + 1], (float)pos[3 * i + 2], 0.f);
  float4 *dp = nullptr;
  float *dl = nullptr;
  if ((rc = dalloc(c, dp, n * sizeof(float4))) || (rc = dalloc(c, dl, n * fs->nf * 4 * sizeof(float)))) {
    dfree(dp); dfree(dl);
    return rc;
  }
  KParams kp = base_params(c);
  kp.field = fs->k;
  std::vector<float> hl(n * fs->nf * 4);
  bool ok = to_dev(c, dp, hp.data(), n * sizeof(float4)) == cudaSuccess;
  if (ok) {
    far_label_kernel<<<(unsigned)std::min<size_t>((n + 7) / 8, (size_t)c->sm_count * 64), 256, 0, c->stream>>>(
        kp, fs->kinds, fs->nf, n, dp, dl);
    ok = cudaGetLastError() == cudaSuccess && cudaStreamSynchronize(c->stream) == cudaSuccess &&
         to_host(c, hl.data(), dl, hl.size() * sizeof(float)) == cudaSuccess;
  }
  dfree(dp); dfree(dl);
  if (!ok) return fail(c, CCS_ERR_CUDA, "field labels: %s", cudaGetErrorString(cudaGetLastError()));
  for (size_t i = 0; i < hl.size(); i++) labels[i] = hl[i];
  return CCS_OK;
}

int ccs_field_get_weights(ccs_ctx *c, float *table, float *mlp, double *scales) {
  if (!c) return CCS_ERR_INVALID;
  if (!c->field) return fail(c, CCS_ERR_INVALID, "no learned field");
  FieldState *fs = c->field;
  if (cudaSetDevice(c->device) != cudaSuccess) return fail(c, CCS_ERR_CUDA, "cudaSetDevice");
  CK(cudaStreamSynchronize(c->stream));
  const size_t nt = (size_t)FL_LEVELS * fs->rows;
  if (table) CK(to_host(c, table, fs->table, nt * sizeof(float2)));
  if (mlp) {
    std::vector<float> m(NM);
    CK(to_host(c, m.data(), fs->mlp, NM * sizeof(float)));
    // external layout: W3 and b3 with nf rows
    std::memcpy(mlp, m.data(), MO_W3 * sizeof(float));
    std::memcpy(mlp + MO_W3, m.data() + MO_W3, fs->nf * FL_H * sizeof(float));
    std::memcpy(mlp + MO_W3 + fs->nf * FL_H, m.data() + MO_B3, fs->nf * sizeof(float));
  }
  if (scales)
    for (int f = 0; f < fs->nf; f++) { scales[f] = fs->s[f]; scales[fs->nf + f] = fs->gs[f]; }
  return CCS_OK;
}

int ccs_field_set_weights(ccs_ctx *c, const float *table, const float *mlp, const double *scales) {
  if (!c) return CCS_ERR_INVALID;
  if (!c->field) return fail(c, CCS_ERR_INVALID, "no learned field: call ccs_field_setup");
  FieldState *fs = c->field;
  if (scales)
    for (int f = 0; f < 2 * fs->nf; f++)
      if (!(scales[f] > 0)) return fail(c, CCS_ERR_INVALID, "scales must be positive");
  if (cudaSetDevice(c->device) != cudaSuccess) return fail(c, CCS_ERR_CUDA, "cudaSetDevice");
  const size_t nt = (size_t)FL_LEVELS * fs->rows;
  if (table) CK(to_dev(c, fs->table, table, nt * sizeof(float2)));
  if (mlp) {
    std::vector<float> m(NM, 0.f);
    std::memcpy(m.data(), mlp, MO_W3 * sizeof(float));
    std::memcpy(m.data() + MO_W3, mlp + MO_W3, fs->nf * FL_H * sizeof(float));
    std::memcpy(m.data() + MO_B3, mlp + MO_W3 + fs->nf * FL_H, fs->nf * sizeof(float));
    CK(to_dev(c, fs->mlp, m.data(), NM * sizeof(float)));
  }
  if (scales)
    for (int f = 0; f < fs->nf; f++) { fs->s[f] = scales[f]; fs->gs[f] = scales[fs->nf + f]; }
  int rc = pack_inference(c, fs);
  if (rc) return rc;
  CK(cudaStreamSynchronize(c->stream));
  return CCS_OK;
}

int ccs_field_loss_grad(ccs_ctx *c, size_t n, const float *pos, const float *labels, double *loss, float *dtable,
                        float *dmlp) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!c->field) return fail(c, CCS_ERR_INVALID, "no learned field: call ccs_field_setup");
  if (n == 0 || n > (1u << 20) || !pos || !labels) return fail(c, CCS_ERR_INVALID, "1..2^20 samples with labels");
  FieldState *fs = c->field;
  const int B = (int)n;
  if ((rc = ensure_scratch(c, fs, n))) return rc;
  std::vector<float4> hp(n);
  std::vector<int> idx(n);
  for (size_t i = 0; i < n; i++) {
    hp[i] = make_float4(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], 0.f);
    idx[i] = (int)i;
  }
  float4 *dp = nullptr;
  float *dl = nullptr, *dloss = nullptr;
  auto cleanup = [&]() { dfree(dp); dfree(dl); dfree(dloss); };
  if ((rc = dalloc(c, dp, n * sizeof(float4))) || (rc = dalloc(c, dl, n * fs->nf * 4 * sizeof(float))) ||
      (rc = dalloc(c, dloss, sizeof(float)))) {
    cleanup();
    return rc;
  }
  const size_t nt = (size_t)FL_LEVELS * fs->rows;
  bool ok = to_dev(c, dp, hp.data(), n * sizeof(float4)) == cudaSuccess &&
            to_dev(c, dl, labels, n * fs->nf * 4 * sizeof(float)) == cudaSuccess &&
            to_dev(c, fs->bidx, idx.data(), n * sizeof(int)) == cudaSuccess &&
            zero_dev(c, fs->tgrad, nt * 2 * sizeof(unsigned long long)) == cudaSuccess;
  if (ok) {
    rc = grad_step(c, fs, dp, dl, B, dloss);
    ok = rc == CCS_OK && cudaStreamSynchronize(c->stream) == cudaSuccess;
  }
  float hl = 0.f;
  std::vector<float> m(NM);
  ok = ok && to_host(c, &hl, dloss, sizeof(float)) == cudaSuccess &&
       to_host(c, m.data(), fs->mgrad, NM * sizeof(float)) == cudaSuccess;
  if (ok && dtable) {
    std::vector<unsigned long long> g(nt * 2);
    ok = to_host(c, g.data(), fs->tgrad, nt * 2 * sizeof(unsigned long long)) == cudaSuccess;
    for (size_t i = 0; ok && i < nt * 2; i++) dtable[i] = (float)((double)(long long)g[i] / FIX_SCALE);
  }
  if (ok) zero_dev(c, fs->tgrad, nt * 2 * sizeof(unsigned long long));
  cleanup();
  if (!ok) return rc ? rc : fail(c, CCS_ERR_CUDA, "loss gradient: %s", cudaGetErrorString(cudaGetLastError()));
  if (loss) *loss = hl;
  if (dmlp) {
    std::memcpy(dmlp, m.data(), MO_W3 * sizeof(float));
    std::memcpy(dmlp + MO_W3, m.data() + MO_W3, fs->nf * FL_H * sizeof(float));
    std::memcpy(dmlp + MO_W3 + fs->nf * FL_H, m.data() + MO_B3, fs->nf * sizeof(float));
  }
  return CCS_OK;
}

}  // extern "C"
