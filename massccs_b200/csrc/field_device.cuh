// field_device.cuh -- device code of the learned field (the surrogate force
// field of the trajectory engine).  No counterpart in the reference
// (cces-cepid/massccs), which evaluates every force exactly
// (src/Force.cpp:34-1725); the field replaces those sums where it is
// trusted, and the exact evaluation stays everywhere else.
//
// Range separation: every pair term (LJ, Coulomb, the dipole's field) is
// split by a smooth switch S(r) (1 below r_in, 0 above r_out, quintic
// smootherstep between) into a near part S * term, summed exactly over the
// atoms within r_out of the site, and a far part (1 - S) * term, which is a
// smooth function of the site position (no atom closer than r_in
// contributes) and is what the network learns.
//
// Model (the checker is oracle/surrogate.py): a multiresolution hash-grid
// encoding of the site position (16 levels x 2 features, smoothstep blending,
// so the encoding has continuous first derivatives) feeds a ReLU MLP
// 32 -> 64 -> 64 -> nf with per-field output scales.  Fields: the far
// potential of each gas site type (N2: the N atoms and the central charge;
// CO2: O and C; atoms: one) and, with the induced dipole, the three
// components of the far electric field.  Each field's gradient is
// back-propagated through the MLP and the encoding: the far forces are
// conservative, and the far field's gradients give its Jacobian.
//
// Inference arithmetic (identical in both paths below, up to FP32 summation
// order): table and the W1/W2 weights in bfloat16, the MMA inputs (encoded
// features, first hidden layer, the back-propagated vectors) rounded to
// bfloat16, FP32 accumulation, biases, output layer and the final
// contraction with the encoding's Jacobian in FP32.
//
//   lane pass   128 trajectories per CTA: per site, the CTA's 128 rows go
//               through four tcgen05.mma stages (M = 128, BF16 in, FP32 in
//               TMEM) -- z1 = X W1^T, z2 = H W2^T, g1 = G2 W2, g0 = G1 W1 --
//               with the epilogues (bias, ReLU, masks, bf16 packing into the
//               next stage's shared-memory operand) done by each row's own
//               thread from its TMEM lane.
//   warp pass   one trajectory per CTA: each site is evaluated by one warp
//               (two hidden units per lane, vectors exchanged by shuffles).
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

namespace ccs {

constexpr int FL_LEVELS = 16;              // hash-grid levels
constexpr int FL_FEAT = 2;                 // features per level
constexpr int FL_E = FL_LEVELS * FL_FEAT;  // encoded features (32)
constexpr int FL_H = 64;                   // hidden width
constexpr int FL_NF = 5;                   // most output fields (2 site types + 3 field components)
constexpr int FL_SITE_FIELDS = 4;          // most fields evaluated at one site (the dipole site)

// Offsets (floats) of the FP32 copies of the (bf16-rounded) MLP in FieldK::mlp.
constexpr int FO_W1 = 0;                          // W1  [64][32]
constexpr int FO_W1T = FO_W1 + FL_H * FL_E;       // W1t [32][64]
constexpr int FO_W2 = FO_W1T + FL_E * FL_H;       // W2  [64][64]
constexpr int FO_W2T = FO_W2 + FL_H * FL_H;       // W2t [64][64]
constexpr int FO_B1 = FO_W2T + FL_H * FL_H;       // b1  [64]
constexpr int FO_B2 = FO_B1 + FL_H;               // b2  [64]
constexpr int FO_W3 = FO_B2 + FL_H;               // w3  [FL_NF][64] (FP32, not rounded)
constexpr int FO_B3 = FO_W3 + FL_NF * FL_H;       // b3  [FL_NF]
constexpr int FO_S = FO_B3 + FL_NF;               // s   [FL_NF] output scales
constexpr int FO_TOTAL = FO_S + FL_NF;

// Byte offsets of the tcgen05 B-operand images in FieldK::umma (each in the
// K-major no-swizzle core-matrix layout: element (row n, k) at
// (k / 8) * (N * 16) + n * 16 + (k % 8) * 2).
constexpr int FU_W1 = 0;                          // W1 : N = 64, K = 32
constexpr int FU_W2 = FU_W1 + FL_H * FL_E * 2;    // W2 : N = 64, K = 64
constexpr int FU_W2T = FU_W2 + FL_H * FL_H * 2;   // W2t: N = 64, K = 64
constexpr int FU_W1T = FU_W2T + FL_H * FL_H * 2;  // W1t: N = 32, K = 64
constexpr int FU_BYTES = FU_W1T + FL_E * FL_H * 2;

// Launch parameters of the learned field (part of KParams; on == 0: off).
struct FieldK {
  const uint32_t *table;       // [FL_LEVELS][1 << log2t] rows of two bf16 features (feature 0 low)
  const uint32_t *exact_bits;  // one bit per voxel: 1 = evaluate this position exactly
  const float *mlp;            // FO_TOTAL floats
  const uint4 *umma;           // FU_BYTES of operand images
  float lo[3];                 // domain cube corner (A)
  float side;                  // domain cube edge (A)
  float scale[FL_LEVELS];      // res_l / side: grid units per A
  int res[FL_LEVELS];
  int dense[FL_LEVELS];        // 1: rows indexed directly, 0: hashed
  uint32_t tmask;              // rows per level - 1
  int log2t;
  float vox_inv;               // 1 / voxel edge of the exact-evaluation bitmap
  int vx, vy, vz;              // bitmap dimensions (voxels from lo)
  float r_in, r_out;           // range separation: the switch runs from r_in to r_out (A)
  int nf;                      // output fields
  int site_field[3];           // far-potential field of each gas site
  int dip_site;                // the induced dipole's site (-1: none)
  int efield;                  // first of the three far-field components (E_x, E_y, E_z)
  int on;
};

// The fields evaluated at site s: its far potential, and at the dipole site
// the three far-field components.  Returns their count.
__device__ __forceinline__ int site_fields(const FieldK &F, int s, int (&fl)[FL_SITE_FIELDS]) {
  fl[0] = F.site_field[s];
  if (s != F.dip_site) return 1;
  fl[1] = F.efield; fl[2] = F.efield + 1; fl[3] = F.efield + 2;
  return 4;
}

// The switch of the range separation and its derivative d/dr.
template <typename T> __device__ __forceinline__ void range_switch(T r, T r_in, T r_out, T &S, T &dS) {
  const T w = r_out - r_in;
  T x = (r - r_in) / w;
  x = x < T(0) ? T(0) : (x > T(1) ? T(1) : x);
  S = T(1) - x * x * x * (T(10) - T(15) * x + T(6) * x * x);
  dS = T(-30) * x * x * (T(1) - x) * (T(1) - x) / w;
}

// ---- exact-evaluation test --------------------------------------------------
// Positions outside the domain, within the fallback radius of an atom, or in
// a voxel whose measured surrogate error exceeds the threshold are evaluated
// exactly (the bitmap holds all three).
__device__ __forceinline__ bool field_exact(const FieldK &F, float x, float y, float z) {
  const int i = (int)floorf((x - F.lo[0]) * F.vox_inv);
  const int j = (int)floorf((y - F.lo[1]) * F.vox_inv);
  const int k = (int)floorf((z - F.lo[2]) * F.vox_inv);
  if (i < 0 || j < 0 || k < 0 || i >= F.vx || j >= F.vy || k >= F.vz) return true;
  const uint32_t v = (uint32_t)i + (uint32_t)F.vx * ((uint32_t)j + (uint32_t)F.vy * (uint32_t)k);
  return (__ldg(&F.exact_bits[v >> 5]) >> (v & 31u)) & 1u;
}

__device__ __forceinline__ float bf16r(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }
__device__ __forceinline__ float bf16lo(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf16hi(uint32_t w) { return __uint_as_float(w & 0xffff0000u); }
__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
  const uint32_t lo = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(a));
  const uint32_t hi = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(b));
  return lo | (hi << 16);
}

// Cell of the point on level l: corner c0, smoothstep weights S and their
// derivatives dS (per A) per axis.
__device__ __forceinline__ void field_cell(const FieldK &F, int l, const float (&x)[3], int (&c0)[3], float (&S)[3],
                                           float (&dS)[3]) {
  const float sc = F.scale[l];
  const int r = F.res[l];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const float p = fminf(fmaxf((x[a] - F.lo[a]) * sc, 0.f), (float)r);
    const int c = min((int)floorf(p), r - 1);
    const float f = p - (float)c;
    c0[a] = c;
    S[a] = f * f * (3.f - 2.f * f);
    dS[a] = 6.f * f * (1.f - f) * sc;
  }
}

// Table row of corner (cx, cy, cz) on level l.
__device__ __forceinline__ uint32_t field_row(const FieldK &F, int l, int cx, int cy, int cz) {
  if (F.dense[l]) {
    const uint32_t r = (uint32_t)F.res[l] + 1u;
    return (uint32_t)cx + r * ((uint32_t)cy + r * (uint32_t)cz);
  }
  return ((uint32_t)cx * 1u ^ (uint32_t)cy * 2654435761u ^ (uint32_t)cz * 805459861u) & F.tmask;
}

// Encoded features e (32) and their Jacobian J (32 x 3) at x, one thread.
__device__ __forceinline__ void field_encode(const FieldK &F, const float (&x)[3], float (&e)[FL_E],
                                             float (&J)[FL_E][3]) {
#pragma unroll
  for (int l = 0; l < FL_LEVELS; l++) {
    int c0[3];
    float S[3], dS[3];
    field_cell(F, l, x, c0, S, dS);
    const uint32_t *tl = F.table + ((size_t)l << F.log2t);
    float e0 = 0.f, e1 = 0.f, j0[3] = {0.f, 0.f, 0.f}, j1[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int c = 0; c < 8; c++) {
      const int ox = c & 1, oy = (c >> 1) & 1, oz = (c >> 2) & 1;
      const float wx = ox ? S[0] : 1.f - S[0], wy = oy ? S[1] : 1.f - S[1], wz = oz ? S[2] : 1.f - S[2];
      const float dx = ox ? dS[0] : -dS[0], dy = oy ? dS[1] : -dS[1], dz = oz ? dS[2] : -dS[2];
      const uint32_t v = __ldg(&tl[field_row(F, l, c0[0] + ox, c0[1] + oy, c0[2] + oz)]);
      const float t0 = bf16lo(v), t1 = bf16hi(v);
      const float w = wx * wy * wz, gx = dx * wy * wz, gy = wx * dy * wz, gz = wx * wy * dz;
      e0 += w * t0; e1 += w * t1;
      j0[0] += gx * t0; j0[1] += gy * t0; j0[2] += gz * t0;
      j1[0] += gx * t1; j1[1] += gy * t1; j1[2] += gz * t1;
    }
    e[2 * l] = e0; e[2 * l + 1] = e1;
#pragma unroll
    for (int a = 0; a < 3; a++) { J[2 * l][a] = j0[a]; J[2 * l + 1][a] = j1[a]; }
  }
}

// ---- warp path: one site evaluated by one warp ------------------------------
// Lane l holds feature l (level l / 2) with its Jacobian row, and hidden units
// 2l, 2l + 1.  For each of the nfo fields fl[k]: its value u[k] and minus its
// gradient g[k] (for a potential: the force), in every lane.
__device__ __forceinline__ void field_site_warp(const FieldK &F, const float (&x)[3], int nfo,
                                                const int (&fl)[FL_SITE_FIELDS], float (&u)[FL_SITE_FIELDS],
                                                float (&g)[FL_SITE_FIELDS][3]) {
  const int lane = threadIdx.x & 31;
  constexpr unsigned FULL = 0xffffffffu;
  // encoding: lane l takes level l >> 1, corners 4 (l & 1) .. + 3
  const int lev = lane >> 1, half = lane & 1;
  int c0[3];
  float S[3], dS[3];
  field_cell(F, lev, x, c0, S, dS);
  const uint32_t *tl = F.table + ((size_t)lev << F.log2t);
  float e0 = 0.f, e1 = 0.f, j0[3] = {0.f, 0.f, 0.f}, j1[3] = {0.f, 0.f, 0.f};
#pragma unroll
  for (int cc = 0; cc < 4; cc++) {
    const int c = 4 * half + cc;
    const int ox = c & 1, oy = (c >> 1) & 1, oz = (c >> 2) & 1;
    const float wx = ox ? S[0] : 1.f - S[0], wy = oy ? S[1] : 1.f - S[1], wz = oz ? S[2] : 1.f - S[2];
    const float dx = ox ? dS[0] : -dS[0], dy = oy ? dS[1] : -dS[1], dz = oz ? dS[2] : -dS[2];
    const uint32_t v = __ldg(&tl[field_row(F, lev, c0[0] + ox, c0[1] + oy, c0[2] + oz)]);
    const float t0 = bf16lo(v), t1 = bf16hi(v);
    const float w = wx * wy * wz, gx = dx * wy * wz, gy = wx * dy * wz, gz = wx * wy * dz;
    e0 += w * t0; e1 += w * t1;
    j0[0] += gx * t0; j0[1] += gy * t0; j0[2] += gz * t0;
    j1[0] += gx * t1; j1[1] += gy * t1; j1[2] += gz * t1;
  }
  // both corner halves of a level, then each lane keeps its own feature
  e0 += __shfl_xor_sync(FULL, e0, 1);
  e1 += __shfl_xor_sync(FULL, e1, 1);
#pragma unroll
  for (int a = 0; a < 3; a++) {
    j0[a] += __shfl_xor_sync(FULL, j0[a], 1);
    j1[a] += __shfl_xor_sync(FULL, j1[a], 1);
  }
  const float ek = bf16r(half ? e1 : e0);
  const float Jk[3] = {half ? j1[0] : j0[0], half ? j1[1] : j0[1], half ? j1[2] : j0[2]};
  const float *M = F.mlp;
  // z1 = W1 e + b1 (units 2l, 2l+1)
  float z1a = __ldg(&M[FO_B1 + 2 * lane]), z1b = __ldg(&M[FO_B1 + 2 * lane + 1]);
#pragma unroll 8
  for (int k = 0; k < FL_E; k++) {
    const float xk = __shfl_sync(FULL, ek, k);
    const float2 w = __ldg(reinterpret_cast<const float2 *>(&M[FO_W1T + k * FL_H + 2 * lane]));
    z1a += w.x * xk; z1b += w.y * xk;
  }
  const bool m1a = z1a > 0.f, m1b = z1b > 0.f;
  const float a1a = bf16r(m1a ? z1a : 0.f), a1b = bf16r(m1b ? z1b : 0.f);
  // z2 = W2 a1 + b2
  float z2a = __ldg(&M[FO_B2 + 2 * lane]), z2b = __ldg(&M[FO_B2 + 2 * lane + 1]);
#pragma unroll 8
  for (int j = 0; j < FL_H; j++) {
    const float aj = __shfl_sync(FULL, (j & 1) ? a1b : a1a, j >> 1);
    const float2 w = __ldg(reinterpret_cast<const float2 *>(&M[FO_W2T + j * FL_H + 2 * lane]));
    z2a += w.x * aj; z2b += w.y * aj;
  }
  const bool m2a = z2a > 0.f, m2b = z2b > 0.f;
#pragma unroll 1
  for (int k = 0; k < nfo; k++) {
    const int f = fl[k];
    const float sf = __ldg(&M[FO_S + f]);
    const float w3a = __ldg(&M[FO_W3 + f * FL_H + 2 * lane]), w3b = __ldg(&M[FO_W3 + f * FL_H + 2 * lane + 1]);
    float up = (m2a ? z2a * w3a : 0.f) + (m2b ? z2b * w3b : 0.f);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) up += __shfl_xor_sync(FULL, up, o);
    u[k] = sf * (up + __ldg(&M[FO_B3 + f]));
    // g2 = w3_f * m2 ; g1 = m1 * (W2^T g2) ; g0 = W1^T g1 ; -grad = -s J^T g0
    const float g2a = bf16r(m2a ? w3a : 0.f), g2b = bf16r(m2b ? w3b : 0.f);
    float g1a = 0.f, g1b = 0.f;
#pragma unroll 8
    for (int o = 0; o < FL_H; o++) {
      const float go = __shfl_sync(FULL, (o & 1) ? g2b : g2a, o >> 1);
      const float2 w = __ldg(reinterpret_cast<const float2 *>(&M[FO_W2 + o * FL_H + 2 * lane]));
      g1a += w.x * go; g1b += w.y * go;
    }
    g1a = bf16r(m1a ? g1a : 0.f);
    g1b = bf16r(m1b ? g1b : 0.f);
    float g0 = 0.f;  // feature `lane`
#pragma unroll 8
    for (int i = 0; i < FL_H; i++) {
      const float gi = __shfl_sync(FULL, (i & 1) ? g1b : g1a, i >> 1);
      g0 += __ldg(&M[FO_W1 + i * FL_E + lane]) * gi;
    }
    float fx = g0 * Jk[0], fy = g0 * Jk[1], fz = g0 * Jk[2];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      fx += __shfl_xor_sync(FULL, fx, o);
      fy += __shfl_xor_sync(FULL, fy, o);
      fz += __shfl_xor_sync(FULL, fz, o);
    }
    g[k][0] = -sf * fx; g[k][1] = -sf * fy; g[k][2] = -sf * fz;
  }
}

// ---- tensor-core path (tcgen05) ---------------------------------------------
// Shared memory of one CTA's MLP tiles (dynamic shared memory, 1024-byte
// aligned): A operands of 128 rows, the four B images, the MMA barrier and
// the TMEM base address.
constexpr int TC_ROWS = 128;
constexpr int TC_SA = 0;                                // X  : 128 x 32 bf16 (8 KB)
constexpr int TC_SH = TC_SA + TC_ROWS * FL_E * 2;       // H  : 128 x 64 bf16 (16 KB)
constexpr int TC_SB = TC_SH + TC_ROWS * FL_H * 2;       // B images (FU_BYTES = 24 KB)
constexpr int TC_BAR = TC_SB + FU_BYTES;                // mbarrier (8 B)
constexpr int TC_TMEM = TC_BAR + 8;                     // TMEM base address (4 B)
constexpr int TC_SMEM_BYTES = TC_TMEM + 8;
constexpr int TC_TMEM_COLS = 64;                        // accumulator columns per CTA
// wait limit on one MMA stage (a stage takes microseconds); past it the
// kernel reports the failure and stops
constexpr unsigned long long TC_WAIT_NS = 200000000ull;  // 0.2 s

__device__ __forceinline__ unsigned long long fl_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Instruction descriptor of tcgen05.mma kind::f16: BF16 A and B (K-major),
// FP32 accumulator, M = 128, N = n.
__device__ __forceinline__ constexpr uint32_t tc_idesc(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}
// Shared-memory matrix descriptor, K-major without swizzle: lbo = bytes
// between the two 8-element K chunks of one MMA, sbo = bytes between 8-row
// groups.
__device__ __forceinline__ uint64_t tc_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(done)
      : "r"(bar), "r"(parity)
      : "memory");
  return done != 0;
}

// 16 FP32 columns of this thread's TMEM lane (warp w reads lanes 32w..32w+31).
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// Set-up of a CTA's tensor-core state: TMEM columns (allocated by warp 0),
// the barrier, and the B images copied into shared memory.  All threads call
// it; returns the TMEM base address.
__device__ __forceinline__ uint32_t tc_setup(const FieldK &F, unsigned char *sm) {
  if (threadIdx.x < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(sm + TC_TMEM)),
                 "r"((uint32_t)TC_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(sm + TC_BAR)), "r"(1u) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  const uint4 *src = F.umma;
  uint4 *dst = reinterpret_cast<uint4 *>(sm + TC_SB);
  for (int i = threadIdx.x; i < FU_BYTES / 16; i += blockDim.x) dst[i] = __ldg(&src[i]);
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  return *reinterpret_cast<volatile uint32_t *>(sm + TC_TMEM);
}

__device__ __forceinline__ void tc_teardown(uint32_t tmem) {
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (threadIdx.x < 32)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)TC_TMEM_COLS));
}

// One MMA stage: D (TMEM, N columns) = A (128 x K, at smem offset a_off) x
// B^T (N x K at b_off), issued by thread 0 after every thread's operand
// writes, then waited for by all threads.  Returns false (in every thread)
// if the stage did not complete within the wait limit.
__device__ __forceinline__ bool tc_stage(unsigned char *sm, uint32_t tmem, int a_off, int b_off, int K, int N,
                                         uint32_t &phase) {
  fence_async_smem();  // this thread's generic writes to the operands -> async proxy
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t bar = smem_u32(sm + TC_BAR);
  if (threadIdx.x == 0) {
    const uint32_t a = smem_u32(sm + a_off), b = smem_u32(sm + b_off);
    const uint32_t idesc = tc_idesc(N);
#pragma unroll 1
    for (int k = 0; k < K; k += 16) {
      // K-chunk pair k/8, k/8 + 1: A chunk stride 128 rows x 16 B, B chunk stride N x 16 B
      const uint64_t ad = tc_desc(a + (uint32_t)(k / 8) * (TC_ROWS * 16), TC_ROWS * 16, 128);
      const uint64_t bd = tc_desc(b + (uint32_t)(k / 8) * (N * 16), N * 16, 128);
      tc_mma(tmem, ad, bd, idesc, k > 0 ? 1u : 0u);
    }
    tc_commit(bar);
  }
  bool done = mbar_try(bar, phase);
  if (!done) {
    const unsigned long long t0 = fl_ns();
#pragma unroll 1
    for (uint32_t it = 1; !done; it++) {
      done = mbar_try(bar, phase);
      if (!done && (it & 255u) == 0 && fl_ns() - t0 > TC_WAIT_NS) break;
    }
  }
  phase ^= 1u;
  const bool all = __syncthreads_and(done) != 0;
  tc_fence_after();
  return all;
}

// Writes a row of N (multiple of 8) bf16 values into the K-major core-matrix
// layout of a 128-row A operand at smem offset off.
template <int N>
__device__ __forceinline__ void tc_store_row(unsigned char *sm, int off, int row, const uint32_t (&packed)[N / 2]) {
#pragma unroll
  for (int c = 0; c < N / 8; c++) {
    uint4 v = make_uint4(packed[4 * c], packed[4 * c + 1], packed[4 * c + 2], packed[4 * c + 3]);
    *reinterpret_cast<uint4 *>(sm + off + c * (TC_ROWS * 16) + row * 16) = v;
  }
}

// The whole MLP of one site position for the CTA's 128 rows (row =
// threadIdx.x), for the nfo fields fl[] (the same in every row): forward
// once, then one backward chain per field.  use: this row holds a position
// to evaluate (others contribute zero rows); e/J: its encoding and Jacobian.
// Out: u[k] and minus the gradient g[k] of field fl[k].  Returns false if an
// MMA stage timed out (the caller stops the kernel).
__device__ __forceinline__ bool tc_site(const FieldK &F, unsigned char *sm, uint32_t tmem, uint32_t &phase,
                                        bool use, const float (&e)[FL_E], const float (&J)[FL_E][3], int nfo,
                                        const int (&fl)[FL_SITE_FIELDS], float (&u)[FL_SITE_FIELDS],
                                        float (&g)[FL_SITE_FIELDS][3]) {
  const int row = threadIdx.x;
  const uint32_t trow = tmem + ((uint32_t)(threadIdx.x & ~31) << 16);  // this warp's TMEM lanes
  const float *M = F.mlp;
  {
    uint32_t pk[FL_E / 2];
#pragma unroll
    for (int k = 0; k < FL_E / 2; k++) pk[k] = use ? pack_bf16x2(e[2 * k], e[2 * k + 1]) : 0u;
    tc_store_row<FL_E>(sm, TC_SA, row, pk);
  }
  if (!tc_stage(sm, tmem, TC_SA, TC_SB + FU_W1, FL_E, FL_H, phase)) return false;
  // epilogue 1: z1 + b1, mask m1, relu -> H (bf16)
  uint32_t m1 = 0u, m1b = 0u;  // units 0..31, 32..63
  {
    uint32_t pk[FL_H / 2];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      float v[16];
      tc_ld16(trow + 16 * q, v);
#pragma unroll
      for (int i = 0; i < 16; i += 2) {
        const int n = 16 * q + i;
        const float za = v[i] + __ldg(&M[FO_B1 + n]), zb = v[i + 1] + __ldg(&M[FO_B1 + n + 1]);
        const uint32_t bits = (za > 0.f ? 1u : 0u) | (zb > 0.f ? 2u : 0u);
        if (n < 32) m1 |= bits << n; else m1b |= bits << (n - 32);
        pk[n / 2] = pack_bf16x2(fmaxf(za, 0.f), fmaxf(zb, 0.f));
      }
    }
    tc_store_row<FL_H>(sm, TC_SH, row, pk);
  }
  if (!tc_stage(sm, tmem, TC_SH, TC_SB + FU_W2, FL_H, FL_H, phase)) return false;
  // epilogue 2: z2 + b2, mask m2, u_f = s_f (w3_f . relu(z2) + b3_f) for every field
  uint32_t m2 = 0u, m2b = 0u;
  {
    float acc[FL_SITE_FIELDS] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int q = 0; q < 4; q++) {
      float v[16];
      tc_ld16(trow + 16 * q, v);
#pragma unroll
      for (int i = 0; i < 16; i += 2) {
        const int n = 16 * q + i;
        const float za = v[i] + __ldg(&M[FO_B2 + n]), zb = v[i + 1] + __ldg(&M[FO_B2 + n + 1]);
        const uint32_t bits = (za > 0.f ? 1u : 0u) | (zb > 0.f ? 2u : 0u);
        if (n < 32) m2 |= bits << n; else m2b |= bits << (n - 32);
        const float aa = fmaxf(za, 0.f), ab = fmaxf(zb, 0.f);
#pragma unroll
        for (int k = 0; k < FL_SITE_FIELDS; k++)
          if (k < nfo) acc[k] += aa * __ldg(&M[FO_W3 + fl[k] * FL_H + n]) + ab * __ldg(&M[FO_W3 + fl[k] * FL_H + n + 1]);
      }
    }
#pragma unroll
    for (int k = 0; k < FL_SITE_FIELDS; k++)
      if (k < nfo) u[k] = __ldg(&M[FO_S + fl[k]]) * (acc[k] + __ldg(&M[FO_B3 + fl[k]]));
  }
#pragma unroll 1
  for (int k = 0; k < nfo; k++) {
    const int f = fl[k];
    {  // G2 = w3_f * m2 (bf16)
      uint32_t pk[FL_H / 2];
#pragma unroll
      for (int n = 0; n < FL_H; n += 2) {
        const uint32_t mm = n < 32 ? (m2 >> n) : (m2b >> (n - 32));
        pk[n / 2] = pack_bf16x2((mm & 1u) ? __ldg(&M[FO_W3 + f * FL_H + n]) : 0.f,
                                (mm & 2u) ? __ldg(&M[FO_W3 + f * FL_H + n + 1]) : 0.f);
      }
      tc_store_row<FL_H>(sm, TC_SH, row, pk);
    }
    if (!tc_stage(sm, tmem, TC_SH, TC_SB + FU_W2T, FL_H, FL_H, phase)) return false;
    // epilogue 3: G1 = m1 * (W2^T G2) (bf16)
    {
      uint32_t pk[FL_H / 2];
#pragma unroll
      for (int q = 0; q < 4; q++) {
        float v[16];
        tc_ld16(trow + 16 * q, v);
#pragma unroll
        for (int i = 0; i < 16; i += 2) {
          const int n = 16 * q + i;
          const uint32_t mm = n < 32 ? (m1 >> n) : (m1b >> (n - 32));
          pk[n / 2] = pack_bf16x2((mm & 1u) ? v[i] : 0.f, (mm & 2u) ? v[i + 1] : 0.f);
        }
      }
      tc_store_row<FL_H>(sm, TC_SH, row, pk);
    }
    if (!tc_stage(sm, tmem, TC_SH, TC_SB + FU_W1T, FL_H, FL_E, phase)) return false;
    // epilogue 4: g0 = W1^T G1 (32), -grad = -s_f J^T g0
    float fx = 0.f, fy = 0.f, fz = 0.f;
#pragma unroll
    for (int q = 0; q < 2; q++) {
      float v[16];
      tc_ld16(trow + 16 * q, v);
#pragma unroll
      for (int i = 0; i < 16; i++) {
        const int kk = 16 * q + i;
        fx += v[i] * J[kk][0]; fy += v[i] * J[kk][1]; fz += v[i] * J[kk][2];
      }
    }
    const float sf = __ldg(&M[FO_S + f]);
    g[k][0] = -sf * fx; g[k][1] = -sf * fy; g[k][2] = -sf * fz;
  }
  return true;
}

}  // namespace ccs
