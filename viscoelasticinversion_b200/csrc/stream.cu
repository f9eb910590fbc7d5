// stream.cu — the step as one streaming kernel per time step (ISO/VTI, FP32).
//
// The grid is cut into strips of W = 120 own columns; each strip is walked
// down in chunks of P = 4 rows.  A persistent CTA owns a contiguous range of
// (strip, chunk) units — the ranges are equal to within one chunk, so there
// is no wave tail — and marches down its strip(s):
//
//   iteration t:  velocity of chunk t      (own columns + 4-column halo)
//                 stress   of chunk t - 1  (own columns)
//
// Every operand arrives by TMA (cp.async.bulk.tensor) into shared memory
// ahead of use: the stresses of the old state into a 16-row ring (chunk t+2
// is requested while chunks t-1..t+1 are read), the old velocities and the
// density of the next velocity chunk while the stress of this iteration is
// computed, the memory variables and stiffnesses of the stress chunk while
// the velocity of this iteration is computed.  The new velocities live in a
// 12-row ring (the stress stencil reaches 4 rows up and down) and go to HBM
// for the own columns only.  The only z overlap between CTAs is the 8-row
// warm-up at the top of each range; x overlap is the 4-column velocity halo.
//
// HBM traffic per cell and step: the algorithmic 2*N_s + N_m planes (v and
// sigma read once through the ring, written once; M read once and written
// in place; medium read once), plus L2-served halo re-reads.
//
// State ping-pongs between the caller's buffers and the plan's copy (the
// velocity halo reads neighbours' old stresses and velocities, which their
// owners are overwriting), like the fused path; the memory variables are
// read and written by their owner only and stay in place.  CPML psi
// ping-pongs between the plan's two sets.  Bounded mbarrier waits report
// through the plan's error word.
#include <atomic>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "fused.cuh"
#include "fused_tma.cuh"
#include "pdl.cuh"
#include "plan.cuh"
#include "stream.cuh"
#include "tma.cuh"
#include "vec.cuh"

namespace vb {

namespace {

constexpr int kW = 120, kP = 4, kNT = 128;  // velocity: (W + 8) / 4 * P = 128 groups
constexpr int kSW = kW + 16;  // sigma ring width: columns x0-8 .. x0+W+8
constexpr int kVW = kW + 8;   // velocity width: columns x0-4 .. x0+W+4
constexpr int kRW = kW + 12;  // rho box: columns x0-4 .. x0+W+8, P+1 rows
constexpr int kCW = kW + 4;   // C55 box: columns x0 .. x0+W+4, P+1 rows
constexpr int kSR = 16;       // sigma ring rows (4 chunks)
constexpr int kVR = 12;       // new-velocity ring rows (3 chunks)
constexpr int kVG = kVW / 4;  // 4-column velocity groups per row (34)

constexpr int r128(int floats) { return (floats * 4 + 127) / 128 * 32; }

template <int KIND, int NSLS>
struct SLayout {
  static constexpr int NM = 3 * NSLS;
  static constexpr int NC = (KIND == VI_MEDIUM_ISO ? 1 : 3) + (NSLS > 0 ? 1 : 0);  // C13 [C11 C33] [tau]
  // float offsets after the barrier block (128 B)
  static constexpr int O_SIG = 32;
  static constexpr int O_VN = O_SIG + r128(3 * kSR * kSW);
  static constexpr int O_VO = O_VN + r128(2 * kVR * kVW);
  static constexpr int O_RHO = O_VO + r128(2 * kP * kVW);
  static constexpr int O_M = O_RHO + r128((kP + 1) * kRW);
  static constexpr int O_C = O_M + (NM > 0 ? r128(NM * kP * kW) : 0);
  static constexpr int O_C55 = O_C + r128(NC * kP * kW);
  static constexpr int FLOATS = O_C55 + r128((kP + 1) * kCW);
  static constexpr int BYTES = FLOATS * 4;
  static constexpr int TX_SIG = 3 * kP * kSW * 4;
  static constexpr int TX_VEL = (2 * kP * kVW + (kP + 1) * kRW) * 4;
  static constexpr int TX_STR = (NM * kP * kW + NC * kP * kW + (kP + 1) * kCW) * 4;
};

__device__ __forceinline__ int vrow(int g) { return (g + 3 * kVR) % kVR; }  // g >= -4

}  // namespace

// One unit = (strip, stress chunk); CTA b owns units [b*Q/G, (b+1)*Q/G).
template <int KIND, int NSLS>
__global__ void __launch_bounds__(kNT, 3)
    k_stream(const StepArgs<float> a, const StreamExtras x, const __grid_constant__ StreamMaps maps) {
  using LY = SLayout<KIND, NSLS>;
  constexpr int NM = LY::NM;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t *bar_sig = reinterpret_cast<uint64_t *>(smem_raw);  // 4 ring slots
  uint64_t *bar_vel = bar_sig + 4, *bar_str = bar_sig + 5;
  float *sm = reinterpret_cast<float *>(smem_raw);
  float *s_sig = sm + LY::O_SIG, *s_vn = sm + LY::O_VN, *s_vo = sm + LY::O_VO, *s_rho = sm + LY::O_RHO;
  float *s_m = sm + LY::O_M, *s_c = sm + LY::O_C, *s_c55 = sm + LY::O_C55;
  const int tid = threadIdx.x;
  const int nx = a.nx, nz = a.nz, xe = nx - L, ze = nz - L;
  const float dt = a.dt;

  pdl_wait();  // the previous step is complete and visible
  if (tid == 0) {
    for (int k = 0; k < 6; ++k) mbar_init(&bar_sig[k], 1);
    for (int k = 0; k < 12; ++k) prefetch_tensormap(&maps.t[k]);
  }
  __syncthreads();

  const long long Q = (long long)x.nstrips * x.nchunks;
  long long u0 = Q * blockIdx.x / gridDim.x;
  const long long u1 = Q * (blockIdx.x + 1) / gridDim.x;
  // sequence numbers of the loads of each barrier group, kept by every
  // thread (the loads are issued and consumed in the same fixed order)
  uint32_t sig_base = 0;  // sigma-ring loads of the previous pieces
  uint32_t nvel = 0, nstr = 0;  // velocity / stress stages consumed so far
  int c0 = 0;

  auto sig_seq = [&](int c) { return sig_base + (uint32_t)(c - (c0 - 2)); };
  auto issue_sig = [&](int x0, int c) {  // chunk c of the old stresses into the ring
    uint64_t *b = &bar_sig[sig_seq(c) & 3];
    const int row0 = L + kP * c;
    float *dst = s_sig + ((kP * c) & (kSR - 1)) * kSW;
    mbar_arrive_expect_tx(b, LY::TX_SIG);
    tma_load_2d(dst, &maps.t[0], x0 - 8, row0, b);
    tma_load_2d(dst + kSR * kSW, &maps.t[1], x0 - 8, row0, b);
    tma_load_2d(dst + 2 * kSR * kSW, &maps.t[2], x0 - 8, row0, b);
  };
  auto issue_vel = [&](int x0, int c) {  // old v and rho of velocity chunk c
    const int row0 = L + kP * c;
    mbar_arrive_expect_tx(bar_vel, LY::TX_VEL);
    tma_load_2d(s_vo, &maps.t[3], x0 - 4, row0, bar_vel);
    tma_load_2d(s_vo + kP * kVW, &maps.t[4], x0 - 4, row0, bar_vel);
    tma_load_2d(s_rho, &maps.t[5], x0 - 4, row0, bar_vel);
  };
  auto issue_str = [&](int x0, int c) {  // M and stiffnesses of stress chunk c
    const int row0 = L + kP * c;
    mbar_arrive_expect_tx(bar_str, LY::TX_STR);
    if constexpr (NM > 0) tma_load_3d(s_m, &maps.t[6], x0, row0, 0, bar_str);
#pragma unroll
    for (int k = 0; k < LY::NC; ++k) tma_load_2d(s_c + k * kP * kW, &maps.t[7 + k], x0, row0, bar_str);
    tma_load_2d(s_c55, &maps.t[11], x0, row0, bar_str);
  };
  // a wait gave up: flag it, then give the loads in flight a bounded time
  // to land before the CTA's shared memory is released
  auto fail = [&](int t, int c1) {
    if (tid != 0) return;
    atomicExch(x.err, 1);
    for (int c = t - 1; c <= t + 2 && c <= c1 + 1; ++c) {
      const uint32_t q = sig_seq(c);
      mbar_wait_bounded(&bar_sig[q & 3], (q >> 2) & 1, 1u << 20);
    }
    mbar_wait_bounded(bar_vel, nvel & 1, 1u << 20);
    mbar_wait_bounded(bar_str, nstr & 1, 1u << 20);
  };
  constexpr uint32_t kTries = 1u << 22;

  while (u0 < u1) {
    // ---- one piece: strip s, stress chunks [c0, c1)
    const int s = (int)(u0 / x.nchunks);
    c0 = (int)(u0 % x.nchunks);
    const long long crem = c0 + (u1 - u0);
    const int c1 = crem < x.nchunks ? (int)crem : x.nchunks;
    u0 += c1 - c0;
    const int x0 = L + kW * s;
    const int *coff = x.chunk_off + (long long)s * (x.nchunks + 1);
    if (tid == 0) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue_sig(x0, c0 - 2);
      issue_sig(x0, c0 - 1);
      issue_sig(x0, c0);
      issue_vel(x0, c0 - 1);
    }
    for (int t = c0 - 1; t <= c1; ++t) {
      if (tid == 0) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        if (t + 2 <= c1 + 1) issue_sig(x0, t + 2);
        if (t >= c0 + 1) issue_str(x0, t - 1);
      }
      // ---- velocity of chunk t (one thread polls the barriers; the CTA
      // barrier then orders everyone's reads after the landed data)
      bool ok = true;
      if (tid == 0) {
#pragma unroll
        for (int d = -1; d <= 1; ++d) {
          const uint32_t q = sig_seq(t + d);
          ok &= mbar_wait_bounded(&bar_sig[q & 3], (q >> 2) & 1, kTries);
        }
        ok &= mbar_wait_bounded(bar_vel, nvel & 1, kTries);
      }
      if (__syncthreads_or(!ok)) {
        fail(t, c1);
        return;
      }
      ++nvel;
      for (int g = tid; g < kP * kVG; g += kNT) {
        const int r = g / kVG, gc = g % kVG;
        const int gi0 = x0 - 4 + 4 * gc, gj = L + kP * t + r;
        const int vb = r * kVW + 4 * gc;
        Q4<float> vxn = lds4(s_vo + vb), vzn = lds4(s_vo + kP * kVW + vb);
        const bool rowin = gj >= L && gj < ze;
        if (rowin && gi0 + 3 >= L && gi0 < xe) {
          // CPML memory of the group, requested before the stencil work
          const int zs = strip_z(gj, nz, a.Tz, a.Bz);
          const bool xstrip = gi0 < a.Lx || gi0 + 3 >= nx - a.Rx;
          const bool own = gi0 >= x0 && gi0 < x0 + kW;
          float pxa[4] = {0, 0, 0, 0}, pxb[4] = {0, 0, 0, 0}, pza[4] = {0, 0, 0, 0}, pzb[4] = {0, 0, 0, 0};
          int xsk[4] = {-1, -1, -1, -1};
          if (xstrip) {
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              xsk[k] = strip_x(gi0 + k, nx, a.Lx, a.Rx);
              if (xsk[k] >= 0) {
                const long long o = (long long)gj * a.wx + xsk[k];
                pxa[k] = a.psix[PX_SXX * a.psix_plane + o];
                pxb[k] = a.psix[PX_SXZ * a.psix_plane + o];
              }
            }
          }
          if (zs >= 0) {
            const long long o = (long long)zs * nx + gi0;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              pza[k] = a.psiz[PZ_SXZ * a.psiz_plane + o + k];
              pzb[k] = a.psiz[PZ_SZZ * a.psiz_plane + o + k];
            }
          }
          // stress taps: ring columns 4gc .. 4gc+11 hold x = gi0-4 .. gi0+7
          const float *sxx_r = s_sig, *szz_r = s_sig + kSR * kSW, *sxz_r = s_sig + 2 * kSR * kSW;
          const int rr = ((kP * t + r) & (kSR - 1)) * kSW;
          float hxx[12], hxz[12];
          row12s(sxx_r + rr + 4 * gc, hxx);
          row12s(sxz_r + rr + 4 * gc, hxz);
          float zxz[4] = {0, 0, 0, 0}, zzz[4] = {0, 0, 0, 0};
#pragma unroll
          for (int q = -4; q <= 4; ++q) {
            const int rq = ((kP * t + r + q) & (kSR - 1)) * kSW + 4 * gc + 4;
            if (q <= 3) {  // ddzm(sxz)
              const float cq = q >= 0 ? a.Dz[q] : -a.Dz[-q - 1];
              const Q4<float> v = q == 0 ? Q4<float>{{hxz[4], hxz[5], hxz[6], hxz[7]}} : lds4(sxz_r + rq);
#pragma unroll
              for (int k = 0; k < 4; ++k) zxz[k] += cq * v.v[k];
            }
            if (q >= -3) {  // ddzp(szz)
              const float cq = q >= 1 ? a.Dz[q - 1] : -a.Dz[-q];
              const Q4<float> v = lds4(szz_r + rq);
#pragma unroll
              for (int k = 0; k < 4; ++k) zzz[k] += cq * v.v[k];
            }
          }
          const Q4<float> r0 = lds4(s_rho + r * kRW + 4 * gc), r1 = lds4(s_rho + (r + 1) * kRW + 4 * gc);
          const float r4 = s_rho[r * kRW + 4 * gc + 4];
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const int gi = gi0 + k;
            if (gi < L || gi >= xe) continue;  // outside the update region: unchanged
            float dxx = dps(hxx, 4 + k, a.Dx), dxxz = dms(hxz, 4 + k, a.Dx);
            float dzxz = zxz[k], dzz = zzz[k];
            if (xstrip) {
              const int xs = xsk[k];
              if (xs >= 0) {
                const float *tb = a.tx;
                const long long o = (long long)gj * a.wx + xs;
                const float p0 = tb[T_BH * nx + gi] * pxa[k] + tb[T_AH * nx + gi] * dxx;
                const float p1 = tb[T_B * nx + gi] * pxb[k] + tb[T_A * nx + gi] * dxxz;
                if (own) {
                  a.psix_o[PX_SXX * a.psix_plane + o] = p0;
                  a.psix_o[PX_SXZ * a.psix_plane + o] = p1;
                }
                dxx = dxx * tb[T_IKH * nx + gi] + p0;
                dxxz = dxxz * tb[T_IK * nx + gi] + p1;
              }
            }
            if (zs >= 0) {
              const float *tb = a.tz;
              const long long o = (long long)zs * nx + gi;
              const float p0 = tb[T_B * nz + gj] * pza[k] + tb[T_A * nz + gj] * dzxz;
              const float p1 = tb[T_BH * nz + gj] * pzb[k] + tb[T_AH * nz + gj] * dzz;
              if (own) {
                a.psiz_o[PZ_SXZ * a.psiz_plane + o] = p0;
                a.psiz_o[PZ_SZZ * a.psiz_plane + o] = p1;
              }
              dzxz = dzxz * tb[T_IK * nz + gj] + p0;
              dzz = dzz * tb[T_IKH * nz + gj] + p1;
            }
            const float rx = k < 3 ? r0.v[k + 1] : r4;
            vxn.v[k] += dt * two_over_fast(r0.v[k] + rx) * (dxx + dzxz);
            vzn.v[k] += dt * two_over_fast(r0.v[k] + r1.v[k]) * (dxxz + dzz);
          }
          // force sources of the velocity columns (own and halo) on this chunk's rows
          const int e0 = t >= 0 && t < x.nchunks ? coff[t] : 0, e1 = t >= 0 && t < x.nchunks ? coff[t + 1] : 0;
          for (int e = e0; e < e1; ++e) {
            const int4 en = x.chunk_ent[e];
            if ((en.w != TL_FORCE_X && en.w != TL_FORCE_Z) || en.y != gj || en.x < gi0 || en.x >= gi0 + 4)
              continue;
            const int k = en.x - gi0;
            const float w = x.it < x.wnt ? x.wavelet[(long long)en.z * x.wnt + x.it] : 0.f;
            const float f = x.amp[en.z] * w;
            if (en.w == TL_FORCE_X)
              add_lane4(vxn, k, dt * two_over_fast(lane4(r0, k) + (k < 3 ? lane4(r0, k + 1) : r4)) * f);
            else
              add_lane4(vzn, k, dt * two_over_fast(lane4(r0, k) + lane4(r1, k)) * f);
          }
          if (own) {
            const long long gg = (long long)gj * nx + gi0;
            stg4(a.vx_o + gg, vxn);
            stg4(a.vz_o + gg, vzn);
            if (x.traces && x.it < x.tnt) {
              for (int e = e0; e < e1; ++e) {
                const int4 en = x.chunk_ent[e];
                if (en.w != TL_RECEIVER || en.y != gj || en.x < gi0 || en.x >= gi0 + 4) continue;
                x.traces[(long long)en.z * x.tnt + x.it] = lane4(vxn, en.x - gi0);
                x.traces[(long long)(x.nrec + en.z) * x.tnt + x.it] = lane4(vzn, en.x - gi0);
              }
            }
          }
        }
        const int vr = vrow(kP * t + r) * kVW + 4 * gc;
        stg4(s_vn + vr, vxn);  // generic store into the shared ring
        stg4(s_vn + kVR * kVW + vr, vzn);
      }
      __syncthreads();  // new velocities of chunk t staged; old-velocity stage free
      if (tid == 0 && t + 1 <= c1) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        issue_vel(x0, t + 1);
      }
      // ---- stress of chunk u = t - 1
      const int u = t - 1;
      if (u >= c0) {
        const bool oks = tid != 0 || mbar_wait_bounded(bar_str, nstr & 1, kTries);
        if (__syncthreads_or(!oks)) {
          fail(t, c1);
          return;
        }
        ++nstr;
        const int r = tid / 32, gc = tid % 32;
        const int gi0 = x0 + 4 * gc, gj = L + kP * u + r;
        if (4 * gc < kW && gi0 < xe && gj < ze) {
          const int e0 = coff[u], e1 = coff[u + 1];
          const int zs = strip_z(gj, nz, a.Tz, a.Bz);
          const bool xstrip = gi0 < a.Lx || gi0 + 3 >= nx - a.Rx;
          float pxa[4] = {0, 0, 0, 0}, pxb[4] = {0, 0, 0, 0}, pza[4] = {0, 0, 0, 0}, pzb[4] = {0, 0, 0, 0};
          int xsk[4] = {-1, -1, -1, -1};
          if (xstrip) {
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              xsk[k] = strip_x(gi0 + k, nx, a.Lx, a.Rx);
              if (xsk[k] >= 0) {
                const long long o = (long long)gj * a.wx + xsk[k];
                pxa[k] = a.psix[PX_VX * a.psix_plane + o];
                pxb[k] = a.psix[PX_VZ * a.psix_plane + o];
              }
            }
          }
          if (zs >= 0) {
            const long long o = (long long)zs * nx + gi0;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              pza[k] = a.psiz[PZ_VZ * a.psiz_plane + o + k];
              pzb[k] = a.psiz[PZ_VX * a.psiz_plane + o + k];
            }
          }
          const float *vx_r = s_vn, *vz_r = s_vn + kVR * kVW;
          const int vb = vrow(kP * u + r) * kVW + 4 * gc;  // columns gi0-4 .. gi0+7
          float hvx[12], hvz[12];
          row12s(vx_r + vb, hvx);
          row12s(vz_r + vb, hvz);
          float zvz[4] = {0, 0, 0, 0}, zvx[4] = {0, 0, 0, 0};
#pragma unroll
          for (int q = -4; q <= 4; ++q) {
            const int rq = vrow(kP * u + r + q) * kVW + 4 * gc + 4;
            if (q <= 3) {  // ddzm(vz)
              const float cq = q >= 0 ? a.Dz[q] : -a.Dz[-q - 1];
              const Q4<float> v = q == 0 ? Q4<float>{{hvz[4], hvz[5], hvz[6], hvz[7]}} : lds4(vz_r + rq);
#pragma unroll
              for (int k = 0; k < 4; ++k) zvz[k] += cq * v.v[k];
            }
            if (q >= -3) {  // ddzp(vx)
              const float cq = q >= 1 ? a.Dz[q - 1] : -a.Dz[-q];
              const Q4<float> v = q == 0 ? Q4<float>{{hvx[4], hvx[5], hvx[6], hvx[7]}} : lds4(vx_r + rq);
#pragma unroll
              for (int k = 0; k < 4; ++k) zvx[k] += cq * v.v[k];
            }
          }
          const bool surf = x.fs && gj == L;
          float rxx[4], rzz[4], rxz[4];
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const int gi = gi0 + k;
            float dxvx = dms(hvx, 4 + k, a.Dx), dxvz = dps(hvz, 4 + k, a.Dx);
            float dzvz = zvz[k], dzvx = zvx[k];
            if (xstrip) {
              const int xs = xsk[k];
              if (xs >= 0) {
                const float *tb = a.tx;
                const long long o = (long long)gj * a.wx + xs;
                const float p0 = tb[T_B * nx + gi] * pxa[k] + tb[T_A * nx + gi] * dxvx;
                const float p1 = tb[T_BH * nx + gi] * pxb[k] + tb[T_AH * nx + gi] * dxvz;
                a.psix_o[PX_VX * a.psix_plane + o] = p0;
                a.psix_o[PX_VZ * a.psix_plane + o] = p1;
                dxvx = dxvx * tb[T_IK * nx + gi] + p0;
                dxvz = dxvz * tb[T_IKH * nx + gi] + p1;
              }
            }
            if (zs >= 0) {
              const float *tb = a.tz;
              const long long o = (long long)zs * nx + gi;
              const float p0 = tb[T_B * nz + gj] * pza[k] + tb[T_A * nz + gj] * dzvz;
              const float p1 = tb[T_BH * nz + gj] * pzb[k] + tb[T_AH * nz + gj] * dzvx;
              a.psiz_o[PZ_VZ * a.psiz_plane + o] = p0;
              a.psiz_o[PZ_VX * a.psiz_plane + o] = p1;
              dzvz = dzvz * tb[T_IK * nz + gj] + p0;
              dzvx = dzvx * tb[T_IKH * nz + gj] + p1;
            }
            rxx[k] = dxvx;
            rzz[k] = dzvz;
            rxz[k] = dzvx + dxvz;
          }
          // own old stresses from the ring (columns gi0.. sit at ring column 8 + 4gc)
          const int sr = ((kP * u + r) & (kSR - 1)) * kSW + 8 + 4 * gc;
          Q4<float> sxx = lds4(s_sig + sr), szz = lds4(s_sig + kSR * kSW + sr), sxz = lds4(s_sig + 2 * kSR * kSW + sr);
          const int cb = r * kW + 4 * gc;
          const Q4<float> c13 = lds4(s_c + cb);
          Q4<float> c11{}, c33{}, tau{};
          if constexpr (KIND != VI_MEDIUM_ISO) {
            c11 = lds4(s_c + kP * kW + cb);
            c33 = lds4(s_c + 2 * kP * kW + cb);
          }
          if constexpr (NSLS > 0) tau = lds4(s_c + (LY::NC - 1) * kP * kW + cb);
          const Q4<float> c55a = lds4(s_c55 + r * kCW + 4 * gc), c55b = lds4(s_c55 + (r + 1) * kCW + 4 * gc);
          const float c55a4 = s_c55[r * kCW + 4 * gc + 4], c55b4 = s_c55[(r + 1) * kCW + 4 * gc + 4];
          Q4<float> m[NM > 0 ? NM : 1];
#pragma unroll
          for (int q = 0; q < NM; ++q) m[q] = lds4(s_m + q * kP * kW + cb);
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            float exx = rxx[k], ezz = rzz[k], exz = rxz[k];
            if constexpr (NSLS > 0) {
              float Sxx = 0, Szz = 0, Sxz = 0;
#pragma unroll
              for (int n = 0; n < NSLS; ++n) {
                Sxx += m[0 * NSLS + n].v[k];
                Szz += m[1 * NSLS + n].v[k];
                Sxz += m[2 * NSLS + n].v[k];
              }
              const float tk = tau.v[k], t1 = 1.f + tk;
              exx = t1 * rxx[k] + tk * Sxx;
              ezz = t1 * rzz[k] + tk * Szz;
              exz = t1 * rxz[k] + tk * Sxz;
            }
            const float C13 = c13.v[k];
            const float C11 = KIND == VI_MEDIUM_ISO ? C13 + 2.f * c55a.v[k] : c11.v[k];
            const float C33 = KIND == VI_MEDIUM_ISO ? C11 : c33.v[k];
            if (surf) ezz = -(C13 * exx) / C33;
            const float c55r = k < 3 ? c55a.v[k + 1] : c55a4, c55br = k < 3 ? c55b.v[k + 1] : c55b4;
            const float C55h = 0.25f * (c55a.v[k] + c55r + c55b.v[k] + c55br);
            sxx.v[k] += dt * (C11 * exx + C13 * ezz);
            szz.v[k] += dt * (C13 * exx + C33 * ezz);
            sxz.v[k] += dt * (C55h * exz);
          }
          const long long gg = (long long)gj * nx + gi0;
          if constexpr (NSLS > 0) {
#pragma unroll
            for (int n = 0; n < NSLS; ++n) {
              const float a1 = a.a1[n], a2 = a.a2[n];
#pragma unroll
              for (int k = 0; k < 4; ++k) {
                m[0 * NSLS + n].v[k] += dt * (a1 * rxx[k] + a2 * m[0 * NSLS + n].v[k]);
                m[1 * NSLS + n].v[k] =
                    surf ? 0.f : m[1 * NSLS + n].v[k] + dt * (a1 * rzz[k] + a2 * m[1 * NSLS + n].v[k]);
                m[2 * NSLS + n].v[k] += dt * (a1 * rxz[k] + a2 * m[2 * NSLS + n].v[k]);
              }
            }
#pragma unroll
            for (int q = 0; q < NM; ++q) stg4(a.m + q * a.mstride + gg, m[q]);
          }
          for (int e = e0; e < e1; ++e) {
            const int4 en = x.chunk_ent[e];
            if (en.w != TL_EXPLOSIVE || en.y != gj || en.x < gi0 || en.x >= gi0 + 4) continue;
            const float w = x.it < x.wnt ? x.wavelet[(long long)en.z * x.wnt + x.it] : 0.f;
            add_lane4(sxx, en.x - gi0, dt * x.amp[en.z] * w);
            add_lane4(szz, en.x - gi0, dt * x.amp[en.z] * w);
          }
          if (surf) szz = Q4<float>{{0, 0, 0, 0}};
          stg4(a.sxx_o + gg, sxx);
          stg4(a.szz_o + gg, szz);
          stg4(a.sxz_o + gg, sxz);
          if (x.fs) {  // stress images of the new state
            const int k = gj - L;
            if (k >= 1 && k <= L) {
              Q4<float> im;
#pragma unroll
              for (int q = 0; q < 4; ++q) im.v[q] = -szz.v[q];
              stg4(a.szz_o + (long long)(L - k) * nx + gi0, im);
            }
            if (k >= 0 && k < L) {
              Q4<float> im;
#pragma unroll
              for (int q = 0; q < 4; ++q) im.v[q] = -sxz.v[q];
              stg4(a.sxz_o + (long long)(L - 1 - k) * nx + gi0, im);
            }
          }
        }
      }
      __syncthreads();  // ring rows of chunk t-2, the stress stage and sigma slot t-1 are free
    }
    sig_base += (uint32_t)(c1 - c0 + 4);  // sigma chunks c0-2 .. c1+1
  }
}

// ------------------------------------------------------------------- host
bool stream_fits(int kind, int nsls) {
  switch (kind * 8 + nsls) {
#define VB_FIT(K, N) \
  case K * 8 + N:    \
    return SLayout<K, N>::BYTES <= 113 * 1024;
    VB_FIT(VI_MEDIUM_ISO, 0) VB_FIT(VI_MEDIUM_ISO, 1) VB_FIT(VI_MEDIUM_ISO, 2) VB_FIT(VI_MEDIUM_ISO, 3)
    VB_FIT(VI_MEDIUM_ISO, 4) VB_FIT(VI_MEDIUM_ISO, 5) VB_FIT(VI_MEDIUM_VTI, 0) VB_FIT(VI_MEDIUM_VTI, 1)
    VB_FIT(VI_MEDIUM_VTI, 2) VB_FIT(VI_MEDIUM_VTI, 3) VB_FIT(VI_MEDIUM_VTI, 4) VB_FIT(VI_MEDIUM_VTI, 5)
#undef VB_FIT
    default:
      return false;
  }
}

template <int KIND, int NSLS>
static int launch_stream_k(const StepArgs<float> &a, const StreamExtras &x, const StreamMaps &m, int nsm,
                           cudaStream_t st, bool pdl) {
  using LY = SLayout<KIND, NSLS>;
  static std::atomic<unsigned long long> attr_set{0};  // one bit per device set up (any thread)
  static std::atomic<int> grid_per_dev[64];  // zero-initialised; any thread
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 64) return set_error(VI_ERR_ARG, "device ordinal out of range");
  if (!(attr_set & (1ULL << dev))) {
    cudaError_t e = cudaFuncSetAttribute(k_stream<KIND, NSLS>, cudaFuncAttributeMaxDynamicSharedMemorySize, LY::BYTES);
    if (e != cudaSuccess) return cuda_check(e, "stream smem attribute");
    int per = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_stream<KIND, NSLS>, kNT, LY::BYTES);
    if (e != cudaSuccess) return cuda_check(e, "stream occupancy");
    grid_per_dev[dev].store(std::max(per, 1) * nsm);
    attr_set |= 1ULL << dev;
  }
  const long long units = (long long)x.nstrips * x.nchunks;
  const int grid = (int)std::min<long long>(grid_per_dev[dev].load(), units);
  return cuda_check(launch_pdl(k_stream<KIND, NSLS>, dim3(grid), dim3(kNT), (size_t)LY::BYTES, st, pdl, a, x, m),
                    "stream launch");
}

static int launch_stream(int kind, int nsls, const StepArgs<float> &a, const StreamExtras &x,
                         const StreamMaps &m, int nsm, cudaStream_t st, bool pdl) {
#define VB_CASE(K, N) \
  if (kind == K && nsls == N) return launch_stream_k<K, N>(a, x, m, nsm, st, pdl);
#define VB_KIND(K) VB_CASE(K, 0) VB_CASE(K, 1) VB_CASE(K, 2) VB_CASE(K, 3) VB_CASE(K, 4) VB_CASE(K, 5)
  VB_KIND(VI_MEDIUM_ISO)
  VB_KIND(VI_MEDIUM_VTI)
#undef VB_KIND
#undef VB_CASE
  return set_error(VI_ERR_ARG, "the streaming step covers ISO and VTI media");
}

static bool al16(const void *q) { return ((uintptr_t)q & 15) == 0; }

bool stream_eligible(const vi_plan *p, const StepArgs<float> &a) {
  const vi_config &c = p->cfg;
  if (c.precision != VI_F32 || c.medium == VI_MEDIUM_TTI || c.nx % 4 != 0) return false;
  if (!stream_fits(c.medium, c.nsls)) return false;
  if (c.free_surface && c.nz - 2 * L < L + 1) return false;
  const void *ptrs[] = {a.vx, a.vz, a.sxx, a.szz, a.sxz, a.rho, a.c11, a.c13, a.c33, a.c55, a.tau, a.m};
  for (const void *q : ptrs)
    if (q && !al16(q)) return false;
  if (c.nsls > 0 && (a.mstride * 4) % 16 != 0) return false;
  return true;
}

// Per-(strip, chunk) source / receiver lists: force sources of the strip's
// velocity columns (own + 4-column halo), explosive sources and receivers of
// its own columns, bucketed by the 4-row chunk of their row.
static void chunk_lists(const vi_config &c, int nstrips, int nchunks, const vi_shot *s,
                        std::vector<int> &off, std::vector<int4> &ent) {
  const int nb = nstrips * (nchunks + 1);
  std::vector<std::vector<int4>> per(nb);
  auto bucket = [&](int strip, int j) { return strip * (nchunks + 1) + (j - L) / kP; };
  auto strip_of = [&](int i) { return (i - L) / kW; };
  if (s) {
    for (int q = 0; q < s->nsrc; ++q) {
      const vi_source &v = s->src_host[q];
      if (v.kind == VI_SRC_EXPLOSIVE) {
        per[bucket(strip_of(v.i), v.j)].push_back(make_int4(v.i, v.j, q, TL_EXPLOSIVE));
        continue;
      }
      const int kind = v.kind == VI_SRC_FORCE_X ? TL_FORCE_X : TL_FORCE_Z;
      for (int b = 0; b < nstrips; ++b) {
        const int x0 = L + kW * b;
        if (v.i >= x0 - 4 && v.i < x0 + kW + 4) per[bucket(b, v.j)].push_back(make_int4(v.i, v.j, q, kind));
      }
    }
    for (int r = 0; r < s->nrec; ++r) {
      const vi_receiver &v = s->rec_host[r];
      per[bucket(strip_of(v.i), v.j)].push_back(make_int4(v.i, v.j, r, TL_RECEIVER));
    }
  }
  off.assign(nb + 1, 0);
  ent.clear();
  for (int b = 0; b < nb; ++b) {
    off[b] = (int)ent.size();
    ent.insert(ent.end(), per[b].begin(), per[b].end());
  }
  off[nb] = (int)ent.size();
}

int stream_steps(vi_plan *p, StepArgs<float> a, const vi_shot *s, int it0, int nsteps, cudaStream_t st) {
  const vi_config &c = p->cfg;
  if (!stream_eligible(p, a))
    return set_error(VI_ERR_ARG,
                     "streaming step needs FP32, an ISO/VTI medium, nx % 4 == 0 and 16-byte aligned planes");
  if (nsteps == 0) return VI_OK;
  const size_t np = (size_t)c.nx * c.nz;
  // second copy of v and sigma, zero outside the update region
  const int nstate = 5 + 3 * c.nsls;
  if (!p->alt) {
    size_t have = 0;
    int rc = ensure_buffer(p, &p->alt, &have, nstate * np * sizeof(float));
    if (rc) return rc;
    rc = cuda_check(cudaMemsetAsync(p->alt, 0, nstate * np * sizeof(float), st), "zero alt state");
    if (rc) return rc;
  }
  const int nstrips = (c.nx - 2 * L + kW - 1) / kW;
  const int nchunks = (c.nz - 2 * L + kP - 1) / kP;
  std::vector<int> off;
  std::vector<int4> ent;
  chunk_lists(c, nstrips, nchunks, s, off, ent);
  int *d_off = nullptr;
  int4 *d_ent = nullptr;
  int rc = stage_tile_lists(p, off, ent, st, &d_off, &d_ent);
  if (rc) return rc;
  float *user[5] = {a.vx, a.vz, a.sxx, a.szz, a.sxz};
  float *alt = (float *)p->alt;
  float *alt_st[5];
  for (int q = 0; q < 5; ++q) alt_st[q] = alt + q * np;
  // tensor maps: parity 0 reads the caller's buffers, parity 1 the plan's copy
  const int e = 4, nx = c.nx, nz = c.nz;
  StreamMaps maps[2];
  const int NC = (c.medium == VI_MEDIUM_ISO ? 1 : 3) + (c.nsls > 0 ? 1 : 0);
  for (int par = 0; par < 2; ++par) {
    float *const *in = par == 0 ? user : alt_st;
    StreamMaps &m = maps[par];
    if ((rc = encode_map(&m.t[0], in[2], e, nx, nz, 1, 0, kSW, kP, 1))) return rc;
    if ((rc = encode_map(&m.t[1], in[3], e, nx, nz, 1, 0, kSW, kP, 1))) return rc;
    if ((rc = encode_map(&m.t[2], in[4], e, nx, nz, 1, 0, kSW, kP, 1))) return rc;
    if ((rc = encode_map(&m.t[3], in[0], e, nx, nz, 1, 0, kVW, kP, 1))) return rc;
    if ((rc = encode_map(&m.t[4], in[1], e, nx, nz, 1, 0, kVW, kP, 1))) return rc;
    if ((rc = encode_map(&m.t[5], a.rho, e, nx, nz, 1, 0, kRW, kP + 1, 1))) return rc;
    if (c.nsls > 0) {
      if ((rc = encode_map(&m.t[6], a.m, e, nx, nz, 3 * c.nsls, a.mstride, kW, kP, 3 * c.nsls))) return rc;
    } else {
      m.t[6] = m.t[5];
    }
    const float *cs[4];
    int n = 0;
    cs[n++] = a.c13;
    if (c.medium != VI_MEDIUM_ISO) {
      cs[n++] = a.c11;
      cs[n++] = a.c33;
    }
    if (c.nsls > 0) cs[n++] = a.tau;
    for (int k = 0; k < 4; ++k) {
      if (k < NC) {
        if ((rc = encode_map(&m.t[7 + k], cs[k], e, nx, nz, 1, 0, kW, kP, 1))) return rc;
      } else {
        m.t[7 + k] = m.t[7];
      }
    }
    if ((rc = encode_map(&m.t[11], a.c55, e, nx, nz, 1, 0, kCW, kP + 1, 1))) return rc;
  }
  StreamExtras x;
  x.nstrips = nstrips;
  x.nchunks = nchunks;
  x.fs = c.free_surface;
  x.chunk_off = d_off;
  x.chunk_ent = d_ent;
  x.amp = (const float *)p->damp;
  x.wavelet = (s && s->nsrc) ? (const float *)s->wavelet_dev : nullptr;
  x.wnt = (s && s->nsrc) ? s->wavelet_nt : 0;
  x.traces = (s && s->nrec) ? (float *)s->traces_dev : nullptr;
  x.tnt = (s && s->nrec) ? s->traces_nt : 0;
  x.nrec = s ? s->nrec : 0;
  x.err = (int *)p->errflag;
  float *psix0 = (float *)p->psix, *psiz0 = (float *)p->psiz;
  for (int k = 0; k < nsteps; ++k) {
    const bool from_user = (k % 2) == 0;
    float *const *in = from_user ? user : alt_st;
    float *const *out = from_user ? alt_st : user;
    a.vx = in[0]; a.vz = in[1]; a.sxx = in[2]; a.szz = in[3]; a.sxz = in[4];
    a.vx_o = out[0]; a.vz_o = out[1]; a.sxx_o = out[2]; a.szz_o = out[3]; a.sxz_o = out[4];
    const int cur = p->psi_cur;
    a.psix = psix0 ? psix0 + cur * kPsiPerSet * p->psix_plane : nullptr;
    a.psix_o = psix0 ? psix0 + (1 - cur) * kPsiPerSet * p->psix_plane : nullptr;
    a.psiz = psiz0 ? psiz0 + cur * kPsiPerSet * p->psiz_plane : nullptr;
    a.psiz_o = psiz0 ? psiz0 + (1 - cur) * kPsiPerSet * p->psiz_plane : nullptr;
    x.it = it0 + k;
    rc = launch_stream(c.medium, c.nsls, a, x, maps[from_user ? 0 : 1], p->nsm, st, k > 0);
    if (rc) return rc;
    p->psi_cur = 1 - cur;
  }
  if (nsteps % 2 == 1) {  // the result sits in the plan's copy
    for (int q = 0; q < 5; ++q) {
      rc = cuda_check(cudaMemcpyAsync(user[q], alt_st[q], np * sizeof(float), cudaMemcpyDeviceToDevice, st),
                      "copy back fields");
      if (rc) return rc;
    }
  }
  return VI_OK;
}

}  // namespace vb
