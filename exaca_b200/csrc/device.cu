// B200 kernels and pool runtime for ExaCA's per-cycle cellular-automaton update.
//
// One CA cycle (src/runCA.cpp:290-341; src/CAupdate.cpp:67-728) is a start and two passes over a
// pool of domains:
//   begin_cycle: per domain, the device-side termination check, cycle/epoch advance and nucleation
//          of the sites whose time has come (nuclei are pre-sorted by time, one cursor each).
//   grow/claim: streams the 16-byte records of the active cells (shared compacted list): diagonal
//          growth from the host-built increment table, solidification of cells with no liquid
//          neighbour, and a 64-bit atomicMin claim (epoch, capturer index) on every liquid neighbour
//          the octahedron reaches. Liquid neighbours come from a per-cell mask kept up to date by
//          captures and nucleations; the 26 critical lengths are read only when the diagonal has
//          reached the cached minimum over the liquid neighbours.
//   capture: per claimed cell: capture by the lowest-index claimant (new decentred octahedron, 26
//          critical lengths), mask updates of its active neighbours, and for those the
//          solidification re-check.
// Stretches of cycles run in one persistent cooperative kernel (k_cycles) whose blocks meet at
// bounded grid-wide barriers between the passes; the last block to reach the end of a cycle
// starts the next one. In k_cycles each block runs the claim steps of the records it flagged right
// after its own growth (a shared-memory queue); a grid-wide claim pass runs only in a cycle where
// some block's queue overflowed. The same passes also run as separate kernels (per-pass timing).
// The claim rule reproduces the Kokkos-Serial loop order exactly: serial visits active cells in
// ascending index and captures flip Liquid to Active in place, so the capturer of a cell is the
// lowest-index claimant, and an active cell sees a neighbour as liquid iff it was liquid at the
// start of the cycle and no lower-index cell claimed it. Only cells next to a claimed cell can lose
// their last such neighbour, so only they are re-checked.
//
// Arithmetic follows the reference's types and operation order; this file is compiled with
// -fmad=false so no multiply-add is contracted, and sqrt/division are IEEE round-to-nearest.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <sstream>
#include <stdexcept>
#include <thread>

#include "pool.hpp"

namespace exaca {

#define CUDA_OK(x)                                                                                                     \
    do {                                                                                                               \
        cudaError_t e__ = (x);                                                                                         \
        if (e__ != cudaSuccess)                                                                                        \
            throw DeviceError(std::string("CUDA error ") + cudaGetErrorString(e__) + " at " #x);                     \
    } while (0)

// A direction's components, its opposite and the capture pass's slot order (directions.hpp), read
// from immediates: lanes asking for different directions read no table.
__device__ __forceinline__ int nb_dx(int l) { return (int)((kDirXP >> l) & 1u) - (int)((kDirXM >> l) & 1u); }
__device__ __forceinline__ int nb_dy(int l) { return (int)((kDirYP >> l) & 1u) - (int)((kDirYM >> l) & 1u); }
__device__ __forceinline__ int nb_dz(int l) { return (int)((kDirZP >> l) & 1u) - (int)((kDirZM >> l) & 1u); }
__device__ __forceinline__ unsigned int field5(unsigned long long a, unsigned long long b, unsigned long long c,
                                               int i) {
    const unsigned long long v = i < 12 ? a : (i < 24 ? b : c);
    const int f = i < 12 ? i : (i < 24 ? i - 12 : i - 24);
    return (unsigned int)(v >> (5 * f)) & 31u;
}
__device__ __forceinline__ int nb_opp(int l) { return (int)field5(kOppA, kOppB, kOppC, l); }
// direction of capture slot s (slots by z, then x, then y); 31 for s >= 26
__device__ __forceinline__ int slot_dir(int s) { return s < 26 ? (int)field5(kSlotA, kSlotB, kSlotC, s) : 31; }

constexpr unsigned int kMaskFresh = 1u << 31; // liquid-neighbour mask not built yet
constexpr unsigned int kMaskDead = 1u << 30;  // solidified by a re-check: leaves the list next cycle
constexpr unsigned int kMaskKeep = 1u << 29;  // this cycle, a neighbour was captured by an index >= this cell's
// the record has been grown (cycle > its CritTimeStep): set by the first growth step, so that the
// capture pass's re-check needs no CritTimeStep (a record's eligibility only changes at a layer
// change, which rebuilds the list)
constexpr unsigned int kMaskGrown = 1u << 28;
constexpr unsigned int kDirBits = (1u << 26) - 1;
constexpr int kErrGrowthTable = 1;
constexpr int kErrListOverflow = 2;
constexpr int kErrBounds = 4;
// One 512-thread block per SM for the persistent kernel (16 warps per SM, 128 registers each): half
// the blocks of two 256-thread ones, so half the arrivals at every grid-wide meeting, and a claim
// step of up to 512 flagged records per block in one round.
constexpr int kBlock = 512;
// rmin2 of a record whose minimum direction is not known: the cached minimum alone applies
constexpr unsigned long long kNoMin2 = 0xffffffffull << 32;

__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; } // std::min
__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; } // std::max

// Number of executed cycles in [1, x]: cycles skipped by the type-S/R jump
// (src/CAupdate.cpp:812-817) are not executed and add no undercooling.
__device__ __forceinline__ long long executed_upto(const DomainDesc &D, long long x) {
    if (x <= 0)
        return 0;
    long long e = x;
    for (int j = 0; j < D.n_jumps; j++) {
        long long lo = D.jump_lo[j], hi = D.jump_hi[j];
        if (x > lo)
            e -= (x < hi ? x : hi) - lo;
    }
    return e;
}

// Block-aggregated reservation of `n` slots per thread on `counter`: one atomicAdd per block. Must
// be called by every thread of the block. Returns this thread's first slot, or ULLONG_MAX on
// overflow (the pool error flag is set).
__device__ __forceinline__ unsigned long long block_reserve_on(unsigned long long *counter, unsigned long long cap,
                                                              int *error, unsigned int n) {
    __shared__ unsigned int s_warp[32];
    __shared__ unsigned long long s_base;
    __shared__ int s_ok;
    // the launch's own warp count (callers launch with different block sizes)
    const unsigned int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, n_warps = blockDim.x >> 5;
    unsigned int incl = n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (unsigned)o)
            incl += v;
    }
    if (lane == 31)
        s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        unsigned int v = lane < n_warps ? s_warp[lane] : 0;
        unsigned int inc2 = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            unsigned int u = __shfl_up_sync(0xffffffffu, inc2, o);
            if (lane >= (unsigned)o)
                inc2 += u;
        }
        if (lane < n_warps)
            s_warp[lane] = inc2 - v;
        unsigned int total = __shfl_sync(0xffffffffu, inc2, n_warps - 1);
        if (lane == 0) {
            unsigned long long b = total ? atomicAdd(counter, (unsigned long long)total) : 0ull;
            s_ok = (b + total <= cap);
            if (!s_ok)
                atomicOr(error, kErrListOverflow);
            s_base = b;
        }
    }
    __syncthreads();
    unsigned long long r = s_ok ? s_base + s_warp[warp] + (incl - n) : ULLONG_MAX;
    __syncthreads(); // s_warp / s_base are reused by the next call
    return r;
}

__device__ __forceinline__ unsigned long long block_reserve(PoolState *P, int slot, unsigned int n) {
    return block_reserve_on(&P->cnt[slot], P->capacity, &P->error, n);
}

// Warp-aggregated reservation (any subset of lanes may call, all with the same counter).
__device__ __forceinline__ unsigned long long warp_reserve(unsigned long long *counter, unsigned long long cap,
                                                           int *error) {
    unsigned int act = __activemask();
    int lane = threadIdx.x & 31;
    int leader = __ffs(act) - 1;
    unsigned long long base = 0;
    if (lane == leader)
        base = atomicAdd(counter, (unsigned long long)__popc(act));
    base = __shfl_sync(act, base, leader);
    unsigned long long r = base + __popc(act & ((1u << lane) - 1));
    if (r >= cap) {
        atomicOr(error, kErrListOverflow);
        return ULLONG_MAX;
    }
    return r;
}

// Block-level sum of per-thread statistics into one shard of the pool counters.
__device__ __forceinline__ void block_stats(PoolState *P, unsigned long long a, unsigned long long b, int ia, int ib) {
    __shared__ unsigned long long s_a[32], s_b[32];
    for (int o = 16; o; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    __syncthreads();
    if ((threadIdx.x & 31) == 0) {
        s_a[threadIdx.x >> 5] = a;
        s_b[threadIdx.x >> 5] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long ta = 0, tb = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
            ta += s_a[w];
            tb += s_b[w];
        }
        int shard = blockIdx.x & (kStatShards - 1);
        if (ta)
            atomicAdd(&P->stat[shard][ia], ta);
        if (tb)
            atomicAdd(&P->stat[shard][ib], tb);
    }
}

__device__ __forceinline__ void cell_coords(const DomainDesc &D, unsigned int c, int &rx, int &ry, int &rz) {
    unsigned int plane = (unsigned int)(D.mx * D.my);
    unsigned int z = c / plane;
    unsigned int rem = c - z * plane;
    unsigned int x = rem / (unsigned int)D.my;
    rz = (int)z;
    rx = (int)x;
    ry = (int)(rem - x * (unsigned int)D.my);
}

// Edge case of src/CAfunctions.cpp:169-213 as a direction mask (ItList, src/CAinitialize.cpp:676-745:
// the edge cases drop the directions leaving the x / y extent, x = 0 before x = mx - 1 and y = 0
// before y = my - 1), restricted to the top of the active window in z (src/CAupdate.cpp:328 checks
// MyNeighborZ < nzActive, window-relative; there is no lower check in the reference, which reads
// one plane below the window; here z >= 0 is kept as a guard).
__device__ __forceinline__ unsigned int edge_mask(int rx, int ry, int rz, int mx, int my, int z_end) {
    unsigned int m = (1u << 26) - 1u;
    m &= ~(ry == 0 ? kDirYM : (ry == my - 1 ? kDirYP : 0u));
    m &= ~(rx == 0 ? kDirXM : (rx == mx - 1 ? kDirXP : 0u));
    if (rz + 1 >= z_end)
        m &= ~kDirZP;
    if (rz - 1 < 0)
        m &= ~kDirZM;
    return m;
}
__device__ __forceinline__ unsigned int neighbour_mask(const DomainDesc &D, int rx, int ry, int rz) {
    return edge_mask(rx, ry, rz, D.mx, D.my, D.z_end);
}

__device__ __forceinline__ int nb_offset(int l, int plane, int my) { return nb_dz(l) * plane + nb_dx(l) * my + nb_dy(l); }

// Fresh octahedron of a newly active cell at its own centre (src/CAupdate.cpp:100-194,
// src/CAinitialize.cpp:1942-2042): DL = 0.01, centre = cell centre, CDL from the orientation table.
__device__ void make_fresh_octahedron(const DomainDesc &D, unsigned int c) {
    int rx, ry, rz;
    cell_coords(D, c, rx, ry, rz);
    int h = D.gid[c];
    int ori = (abs(h) - 1) % 10000;
    if (ori < 0)
        ori += 10000;
    D.dl[c] = 0.01f;
    D.doc[3ull * c + 0] = (float)((double)(rx + D.xoff) + 0.5);
    D.doc[3ull * c + 1] = (float)((double)(ry + D.yoff) + 0.5);
    D.doc[3ull * c + 2] = (float)((double)rz + 0.5);
    const float2 *t = reinterpret_cast<const float2 *>(D.cdl_table + 26 * ori);
    float2 *o = reinterpret_cast<float2 *>(D.cdl + 26ull * c);
#pragma unroll
    for (int n = 0; n < 13; n++)
        o[n] = t[n];
}


__device__ __forceinline__ long long domain_liquid(const DomainDesc &D) {
    long long v = D.liquid;
#pragma unroll
    for (int q = 0; q < kLiquidShards; q++)
        v += __ldcg(&D.liquid_shard[q]);
    return v;
}

// ---------------------------------------------------------------------------------------------
// Capture of liquid cell t by active cell c through neighbour direction l
// (src/CAupdate.cpp:353-563, 713-717).
// Cooperative over kLanes lanes: the group's lanes share the geometry, each independent division
// and square root of a set (the three angles, normal components, distances and direction
// components, the four side lengths, the two projections) evaluated once, on its own lane, with the
// reference's expression, and passed to the others by shuffles; lane `sub` computes critical
// lengths sub, sub + kLanes, ...; lane 0 of the group writes the scalar state. Returns the new
// DiagonalLength. Over the directions in `liq` among the lane's own,
// (mn, d1, mn2) receive the smallest critical length, its lowest direction and the second-smallest
// (+inf and 0xffffffff where there is none), as a claim step's scan would find them.
template <int kLanes>
__device__ float capture_cell(const DomainDesc &D, unsigned int c, unsigned int t, int l, int sub, int h, float docx,
                              float docy, float docz, unsigned int liq, float &mn, unsigned int &d1, float &mn2) {
    int rx, ry, rz;
    cell_coords(D, c, rx, ry, rz);
    const int GlobalX = rx + D.xoff, GlobalY = ry + D.yoff, GlobalZ = rz;
    int ori = (abs(h) - 1) % 10000;
    if (ori < 0)
        ori += 10000;
    const float *g = D.guv + 9 * ori;
    const float g0 = g[0], g1 = g[1], g2 = g[2], g3 = g[3], g4 = g[4], g5 = g[5], g6 = g[6], g7 = g[7], g8 = g[8];
    const double cxold = docx;
    const double cyold = docy;
    const double czold = docz;
    double xp = GlobalX + nb_dx(l) + 0.5;
    double yp = GlobalY + nb_dy(l) + 0.5;
    double zp = GlobalZ + nb_dz(l) + 0.5;
    double x0 = xp - cxold;
    double y0 = yp - cyold;
    double z0 = zp - czold;
    static_assert(kLanes >= 4 && kLanes <= 32, "the geometry spreads over at least four lanes");
    const unsigned int gmask = (kLanes == 32 ? 0xffffffffu : ((1u << kLanes) - 1u))
                               << ((int)(threadIdx.x & 31) / kLanes * kLanes);
    double mag0 = sqrtf((float)(x0 * x0 + y0 * y0 + z0 * z0));
    // Angle1..3 on lanes 0..2 (src/CAupdate.cpp:382-393), their signs by ballot
    const int q3 = sub < 3 ? sub : 0;
    const float ga = q3 == 0 ? g0 : (q3 == 1 ? g3 : g6), gb = q3 == 0 ? g1 : (q3 == 1 ? g4 : g7),
                gc = q3 == 0 ? g2 : (q3 == 1 ? g5 : g8);
    double Angle = (ga * x0 + gb * y0 + gc * z0) / mag0;
    const unsigned int neg = __ballot_sync(gmask, Angle < 0) >> ((int)(threadIdx.x & 31) / kLanes * kLanes);
    float s1 = (float)(2 * (int)(neg & 1u) - 1);
    float s2 = (float)(2 * (int)((neg >> 1) & 1u) - 1);
    float s3 = (float)(2 * (int)((neg >> 2) & 1u) - 1);
    double Diag1X = g0 * s1, Diag1Y = g1 * s1, Diag1Z = g2 * s1;
    double Diag2X = g3 * s2, Diag2Y = g4 * s2, Diag2Z = g5 * s2;
    double Diag3X = g6 * s3, Diag3Y = g7 * s3, Diag3Z = g8 * s3;
    double U1x = Diag2X - Diag1X, U1y = Diag2Y - Diag1Y, U1z = Diag2Z - Diag1Z;
    double U2x = Diag3X - Diag1X, U2y = Diag3Y - Diag1Y, U2z = Diag3Z - Diag1Z;
    double UUx = U1y * U2z - U1z * U2y;
    double UUy = U1z * U2x - U1x * U2z;
    double UUz = U1x * U2y - U1y * U2x;
    double NDem = sqrtf((float)(UUx * UUx + UUy * UUy + UUz * UUz));
    // n0..n2 on lanes 0..2
    const double nq = (q3 == 0 ? UUx : (q3 == 1 ? UUy : UUz)) / NDem;
    double n0 = __shfl_sync(gmask, nq, 0, kLanes), n1 = __shfl_sync(gmask, nq, 1, kLanes),
           n2 = __shfl_sync(gmask, nq, 2, kLanes);
    double ParaT = (n0 * x0 + n1 * y0 + n2 * z0) / (n0 * Diag1X + n1 * Diag1Y + n2 * Diag1Z);
    double TX[3], TY[3], TZ[3];
    TX[0] = cxold + ParaT * Diag1X;
    TY[0] = cyold + ParaT * Diag1Y;
    TZ[0] = czold + ParaT * Diag1Z;
    TX[1] = cxold + ParaT * Diag2X;
    TY[1] = cyold + ParaT * Diag2Y;
    TZ[1] = czold + ParaT * Diag2Z;
    TX[2] = cxold + ParaT * Diag3X;
    TY[2] = cyold + ParaT * Diag3Y;
    TZ[2] = czold + ParaT * Diag3Z;
    // Dist[0..2] on lanes 0..2
    const double tqx = q3 == 0 ? TX[0] : (q3 == 1 ? TX[1] : TX[2]), tqy = q3 == 0 ? TY[0] : (q3 == 1 ? TY[1] : TY[2]),
                 tqz = q3 == 0 ? TZ[0] : (q3 == 1 ? TZ[1] : TZ[2]);
    const float distq =
        sqrtf((float)(((tqx - xp) * (tqx - xp)) + ((tqy - yp) * (tqy - yp)) + ((tqz - zp) * (tqz - zp))));
    double Dist[3];
    Dist[0] = __shfl_sync(gmask, distq, 0, kLanes);
    Dist[1] = __shfl_sync(gmask, distq, 1, kLanes);
    Dist[2] = __shfl_sync(gmask, distq, 2, kLanes);
    int x = (Dist[0] < Dist[1]);
    int y = (Dist[1] < Dist[2]);
    int z = (Dist[2] < Dist[0]);
    int idx = 2 * (z - y) * z + (y - x) * y;
    double mindist = Dist[idx];
    double xc = TX[idx], yc = TY[idx], zc = TZ[idx];
    int i1 = (idx + 1) % 3, i2 = (idx + 2) % 3;
    double x1 = TX[i1], y1 = TY[i1], z1 = TZ[i1];
    double x2 = TX[i2], y2 = TY[i2], z2 = TZ[i2];
    // D1..D4 on lanes 0..3: D1 = |p - v2|, D2 = |c - v2|, D3 = |p - v1|, D4 = |c - v1|
    const int q4 = sub & 3;
    const double ax = (q4 & 1) ? xc : xp, ay = (q4 & 1) ? yc : yp, az = (q4 & 1) ? zc : zp;
    const double bx = (q4 & 2) ? x1 : x2, by = (q4 & 2) ? y1 : y2, bz = (q4 & 2) ? z1 : z2;
    const float dq = sqrtf((float)(((ax - bx) * (ax - bx)) + ((ay - by) * (ay - by)) + ((az - bz) * (az - bz))));
    double D1 = __shfl_sync(gmask, dq, 0, kLanes);
    double D2 = __shfl_sync(gmask, dq, 1, kLanes);
    double D3 = __shfl_sync(gmask, dq, 2, kLanes);
    double D4 = __shfl_sync(gmask, dq, 3, kLanes);
    double I1 = 0, I2 = D2, J1 = 0, J2 = D4;
    if (mindist != 0) {
        // I1 on lane 0, J1 on lane 1
        const bool j = sub & 1;
        const double ex = j ? x1 : x2, ey = j ? y1 : y2, ez = j ? z1 : z2;
        const double Da = j ? D3 : D1, Db = j ? D4 : D2;
        const double ij = Da * ((xp - ex) * (xc - ex) + (yp - ey) * (yc - ey) + (zp - ez) * (zc - ez)) / (Da * Db);
        I1 = __shfl_sync(gmask, ij, 0, kLanes);
        I2 = D2 - I1;
        J1 = __shfl_sync(gmask, ij, 1, kLanes);
        J2 = D4 - J1;
    }
    const double sqrt3 = sqrt(3.0);
    double L12 = 0.5 * (dmin(I1, sqrt3) + dmin(I2, sqrt3));
    double L13 = 0.5 * (dmin(J1, sqrt3) + dmin(J2, sqrt3));
    double NewODiagL = sqrt(2.0) * dmax(L12, L13);
    double cd0 = xc - cxold, cd1 = yc - cyold, cd2 = zc - czold;
    double nd = sqrt(cd0 * cd0 + cd1 * cd1 + cd2 * cd2);
    // uv0..uv2 on lanes 0..2
    const double uvq = (q3 == 0 ? cd0 : (q3 == 1 ? cd1 : cd2)) / nd;
    double uv0 = __shfl_sync(gmask, uvq, 0, kLanes), uv1 = __shfl_sync(gmask, uvq, 1, kLanes),
           uv2 = __shfl_sync(gmask, uvq, 2, kLanes);
    double cx = xc - NewODiagL * uv0;
    double cy = yc - NewODiagL * uv1;
    double cz = zc - NewODiagL * uv2;
    if (sub == 0) {
        D.gid[t] = h;
        D.dl[t] = (float)NewODiagL;
        D.doc[3ull * t + 0] = (float)cx;
        D.doc[3ull * t + 1] = (float)cy;
        D.doc[3ull * t + 2] = (float)cz;
    }
    // face normals: float sums of the unit-vector components (src/CAupdate.cpp:526-551)
    double Fx[4], Fy[4], Fz[4];
    Fx[0] = g0 + g3 + g6;
    Fx[1] = g0 - g3 + g6;
    Fx[2] = g0 + g3 - g6;
    Fx[3] = g0 - g3 - g6;
    Fy[0] = g1 + g4 + g7;
    Fy[1] = g1 - g4 + g7;
    Fy[2] = g1 + g4 - g7;
    Fy[3] = g1 - g4 - g7;
    Fz[0] = g2 + g5 + g8;
    Fz[1] = g2 - g5 + g8;
    Fz[2] = g2 + g5 - g8;
    Fz[3] = g2 - g5 - g8;
#pragma unroll 1
    for (int n = sub; n < 26; n += kLanes) {
        double a0 = xp + nb_dx(n) - cx;
        double b0 = yp + nb_dy(n) - cy;
        double d0 = zp + nb_dz(n) - cz;
        double q0 = a0 * Fx[0] + b0 * Fy[0] + d0 * Fz[0];
        double q1 = a0 * Fx[1] + b0 * Fy[1] + d0 * Fz[1];
        double q2 = a0 * Fx[2] + b0 * Fy[2] + d0 * Fz[2];
        double q3 = a0 * Fx[3] + b0 * Fy[3] + d0 * Fz[3];
        double m = dmax(dmax(fabs(q0), fabs(q1)), dmax(fabs(q2), fabs(q3)));
        const float v = (float)m;
        D.cdl[26ull * t + n] = v;
        if ((liq >> n) & 1u) {
            if (v < mn) {
                mn2 = mn;
                mn = v;
                d1 = (unsigned int)n;
            }
            else if (v < mn2) {
                mn2 = v;
            }
        }
    }
    return (float)NewODiagL;
}

// ---------------------------------------------------------------------------------------------
// Start of a CA cycle (src/runCA.cpp:290-298, src/CAupdate.cpp:67-200): list swap, device-side
// termination check, cycle advance, nucleation. In the persistent kernel the start of a few domains
// runs in one block while the rest of the grid waits, so its cost is its chain of dependent round
// trips to L2 / HBM. Every load that does not depend on an earlier one goes out in the same round:
//   1. the pool's list counters, and each domain's descriptor fields;
//   2. the next 32 nucleation sites by time, with the rest of the descriptor;
//   3. per due site: its CellType, LayerID, GrainID and CritTimeStep;
//   4. per firing site, with the whole warp: its critical-length row and its neighbours' CellTypes and
//      list positions (the list slots of all firing sites are reserved under the first such round).
// Reads that may see data other blocks of the same kernel wrote go through L2 (__ldcg).

// Pool part (warp 0): when `close`, the records the last capture pass appended join the list the
// next cycle reads, which ends the previous cycle; then the list swap, the compaction decision and
// the per-cycle counters. One round of loads. The list this cycle reads goes to *cur_out if given.
__device__ __forceinline__ void lists_start(PoolState *P, bool close, int *cur_out) {
    if (threadIdx.x < 32) {
        static_assert(kShards == 32, "one lane per shard");
        const int lane = threadIdx.x;
        unsigned long long added = __ldcg(&P->tomb_s[lane].v);
        unsigned long long appended = close ? __ldcg(&P->tcnt_s[lane].v) : 0ull;
        int prev = 0, cur = 0;
        unsigned long long cnt0 = 0, cnt1 = 0, tombs = 0, cap = 0;
        if (lane == 0) {
            prev = __ldcg(&P->cur);
            cur = __ldcg(&P->pending);
            cnt0 = __ldcg(&P->cnt[0]);
            cnt1 = __ldcg(&P->cnt[1]);
            tombs = __ldcg(&P->tombs);
            cap = P->capacity;
        }
        P->tomb_s[lane].v = 0;
        P->qcnt_s[lane].v = 0;
        P->tcnt_s[lane].v = 0;
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            added += __shfl_down_sync(0xffffffffu, added, o);
            appended += __shfl_down_sync(0xffffffffu, appended, o);
        }
        if (lane == 0) {
            P->claim_overflow = 0;
            if (close) {
                // the capture pass reserved its new records' slots past the count of list `cur`
                const unsigned long long grown = (cur ? cnt1 : cnt0) + appended;
                if (grown <= cap) {
                    if (cur)
                        cnt1 = grown;
                    else
                        cnt0 = grown;
                    P->cnt[cur] = grown;
                }
            }
            // the list the previous cycle left becomes current; when it was a compacted copy, the old
            // one is emptied and carries no dropped records any more
            const unsigned long long cnt_cur = cur ? cnt1 : cnt0;
            tombs += added;
            if (cur != prev) {
                P->cnt[prev] = 0;
                tombs = 0;
            }
            P->tombs = tombs;
            P->cur = cur;
            // compact when dropped records exceed a quarter of the list (an eighth, and a sixteenth,
            // measured slower: the compaction pass costs more per record than the tombstones it
            // removes)
            const int compact = tombs * 4 > cnt_cur ? 1 : 0;
            P->compact = compact;
            P->pending = compact ? cur ^ 1 : cur;
            if (compact)
                P->cnt[cur ^ 1] = 0;
            if (cur_out)
                *cur_out = cur;
        }
    }
}

__device__ __noinline__ void begin_lists(PoolState *P, bool close) { lists_start(P, close, nullptr); }

constexpr int kSerialDomains = 8; // up to this many domains one block starts each cycle alone

// The domains that had not ended at the last state read, when there are at most kSerialDomains of
// them (a kernel argument, so the cycle start reads their indices without a global round trip;
// the first has the most cells). n < 0: start every domain of the pool.
struct AliveSet {
    int n;
    int idx[kSerialDomains];
};

// Descriptor fields of the first round (the cursor into the nucleation sites and what decides
// whether the domain runs this cycle).
struct DomainStart {
    const int32_t *nuc_time, *nuc_loc;
    int8_t *ctype;
    int done, check_mode, cycle0, cursor0, n_nuclei;
};

__device__ __forceinline__ DomainStart load_start(const DomainDesc &D) {
    DomainStart s;
    s.nuc_time = D.nuc_time;
    s.nuc_loc = D.nuc_loc;
    s.ctype = D.ctype;
    s.n_nuclei = D.n_nuclei;
    s.check_mode = D.check_mode;
    s.done = __ldcg(&D.done);
    s.cycle0 = __ldcg(&D.cycle);
    s.cursor0 = __ldcg(&D.nuc_cursor);
    return s;
}

// Cycle start of domain d by one warp (all lanes call with the same arguments).
__device__ __forceinline__ void start_domain(PoolState *P, DomainDesc &D, const DomainStart &s, unsigned int d,
                                             int cur, unsigned long long &nucleated) {
    const unsigned int lane = threadIdx.x & 31;
    if (s.ctype == nullptr || s.done)
        return;
    if (s.check_mode && s.cycle0 > 0 && s.cycle0 % 1000 == 0 && domain_liquid(D) == 0) {
        // src/CAupdate.cpp:782-783: no superheated or undercooled liquid left
        if (lane == 0)
            D.done = 1;
        return;
    }
    const int cycle = s.cycle0 + 1;
    int cursor = s.cursor0, fired_total = 0;
    // round 2: the rest of the descriptor goes out with the first batch of sites
    const int8_t *const layer = D.layer;
    int32_t *const gid = D.gid;
    const int32_t *const cts_run = D.cts_run;
    float *const dl = D.dl, *const doc = D.doc, *const cdl = D.cdl;
    const float *const cdl_table = D.cdl_table;
    unsigned int *const pos = D.pos;
    const int layer_no = D.layer_no, mx = D.mx, my = D.my, z_end = D.z_end, xoff = D.xoff, yoff = D.yoff;
    const long long active_size = D.active_size;
    const unsigned int epoch0 = __ldcg(&D.epoch);
    const int nn0 = __ldcg(&D.nn);
    const long long liquid0 = __ldcg(&D.liquid);
    // every 64th cycle of a device-terminated domain, in its last phase (every cell past its
    // CritTimeStep), whether any liquid is left: these loads go with this round, and the answer is
    // used after the sites, none of which can fire without liquid
    const bool probe = s.check_mode && (s.cycle0 & 63) == 0;
    const int dry_since = probe ? __ldcg(&D.dry_since) : 0;
    const int cts_max = probe ? D.cts_max : INT_MAX;
    long long dry = probe && lane < kLiquidShards ? __ldcg(&D.liquid_shard[lane]) : 0;
    const unsigned long long cap = P->capacity;
    unsigned int *const rstat = P->rstat[cur];
    // src/CAupdate.cpp:76-198: sites with cycle >= NucleationTimes that are still liquid
    while (cursor < s.n_nuclei) {
        const int idx = cursor + (int)lane;
        const int t = idx < s.n_nuclei ? __ldg(s.nuc_time + idx) : INT_MAX;
        const int l = idx < s.n_nuclei ? __ldg(s.nuc_loc + idx) : -1;
        const bool due = t <= cycle;
        // sites are sorted by time, so the due ones form a prefix
        const int n_due = __popc(__ballot_sync(0xffffffffu, due));
        if (n_due == 0)
            break;
        // round 3
        bool fire = false;
        unsigned int loc = 0;
        int h = 0, cts = 0;
        if (due) {
            if (l < 0 || l >= active_size) {
                atomicOr(&D.error, kErrBounds);
            }
            else {
                loc = (unsigned int)l;
                const int8_t site_type = __ldcg(s.ctype + loc);
                const int site_layer = layer[loc];
                h = __ldcg(gid + loc);
                cts = cts_run[loc];
                fire = site_type == kLiquid && site_layer <= layer_no;
            }
        }
        // list slots of the firing sites (one atomic; it completes under round 4)
        const unsigned long long my_slot = fire ? warp_reserve(&P->cnt[cur], cap, &P->error) : ULLONG_MAX;
        // round 4, one firing site at a time with the whole warp: lanes 0-12 copy the fresh
        // octahedron's critical lengths (src/CAupdate.cpp:100-194), lane n < 26 reads neighbour n's
        // type and list position (an active neighbour drops the site from its liquid mask)
        const int plane = mx * my;
        for (unsigned int todo = __ballot_sync(0xffffffffu, fire); todo; todo &= todo - 1) {
            const int src = __ffs(todo) - 1;
            const unsigned int site = __shfl_sync(0xffffffffu, loc, src);
            const int site_gid = __shfl_sync(0xffffffffu, h, src);
            const unsigned int z = site / (unsigned int)plane;
            const unsigned int rem = site - z * (unsigned int)plane;
            const int rx = (int)(rem / (unsigned int)my), ry = (int)(rem - (unsigned int)rx * (unsigned int)my),
                      rz = (int)z;
            const unsigned int valid = edge_mask(rx, ry, rz, mx, my, z_end);
            int ori = (abs(site_gid) - 1) % 10000;
            if (ori < 0)
                ori += 10000;
            float2 row = make_float2(0.0f, 0.0f);
            if (lane < 13)
                row = reinterpret_cast<const float2 *>(cdl_table + 26 * ori)[lane];
            const bool nb = lane < 26 && ((valid >> lane) & 1u);
            int8_t nb_type = kLiquid;
            unsigned int nb_pos = 0;
            if (nb) {
                const long long a = (long long)site + nb_offset((int)lane, plane, my);
                nb_type = __ldcg(s.ctype + a);
                nb_pos = __ldcg(pos + a);
            }
            const unsigned long long slot = __shfl_sync(0xffffffffu, my_slot, src);
            if (lane < 13)
                reinterpret_cast<float2 *>(cdl + 26ull * site)[lane] = row;
            if (lane == 0) {
                dl[site] = 0.01f;
                doc[3ull * site + 0] = (float)((double)(rx + xoff) + 0.5);
                doc[3ull * site + 1] = (float)((double)(ry + yoff) + 0.5);
                doc[3ull * site + 2] = (float)((double)rz + 0.5);
            }
            if (lane == (unsigned int)src) {
                if (slot != ULLONG_MAX) {
                    ActiveRec r;
                    r.cell = site;
                    r.dl = 0.01f;
                    r.cdl_min = 0.0f;
                    r.cts = cts;
                    P->rec[cur][slot] = r;
                    P->rdom[cur][slot] = d;
                    rstat[slot] = kMaskFresh;
                    P->rmin2[cur][slot] = kNoMin2;
                    pos[site] = (unsigned int)slot;
                }
                s.ctype[site] = kActive;
            }
            if (nb && nb_type == kActive && nb_pos < cap)
                atomicAnd(rstat + nb_pos, ~(1u << nb_opp((int)lane)));
            __syncwarp();
        }
        fired_total += __popc(__ballot_sync(0xffffffffu, fire));
        cursor += n_due;
        if (n_due < 32)
            break;
    }
    bool ended = false;
    if (probe && s.cycle0 - 2 >= cts_max) {
#pragma unroll
        for (int o = 16; o; o >>= 1)
            dry += __shfl_xor_sync(0xffffffffu, dry, o);
        if (dry + liquid0 == 0 && fired_total == 0) {
            if (dry_since == 0) {
                if (lane == 0)
                    D.dry_since = s.cycle0;
            }
            else {
                // At least a whole cycle has run with no liquid and every cell past its CritTimeStep,
                // so every active cell has found no liquid neighbour and solidified
                // (src/CAupdate.cpp:722-725); nothing changes until the next 1000-cycle check, which
                // ends the domain (src/CAupdate.cpp:782-783). It ends here with that check's cycle.
                ended = true;
            }
        }
    }
    if (lane == 0 && ended) {
        D.cycle = (s.cycle0 + 999) / 1000 * 1000;
        D.done = 1;
    }
    else if (lane == 0) {
        D.cycle = cycle;
        D.epoch = epoch0 + 1;
        D.nuc_cursor = cursor;
        D.nn = nn0 + fired_total;
        D.liquid = liquid0 - fired_total;
        nucleated += fired_total;
    }
}

// Cycle start, per-domain part, across the grid: warps first_warp, first_warp + warp_stride, ...
// take one domain each (the current list was settled by begin_lists before a grid-wide meeting).
__device__ __noinline__ void begin_domains(PoolState *P, DomainDesc *desc, int n_domains, int first_warp,
                                           int warp_stride) {
    const int cur = __ldcg(&P->cur);
    unsigned long long nucleated = 0;
    for (int d = first_warp; d < n_domains; d += warp_stride) {
        const DomainStart s = load_start(desc[d]);
        start_domain(P, desc[d], s, (unsigned int)d, cur, nucleated);
    }
    if ((threadIdx.x & 31) == 0 && nucleated)
        atomicAdd(&P->stat[0][kStatNucleated], nucleated);
}

// Cycle start by one block: the pool part in warp 0 while every warp loads its first domain's
// descriptor, then the domains with the block's warps. With `close` it first ends the previous
// cycle (finish_capture).
__device__ __noinline__ void begin_cycle(PoolState *P, bool close, DomainDesc *desc, int n_domains, AliveSet alive) {
    __shared__ int s_cur;
    const int w = (int)(threadIdx.x >> 5), nw = (int)(blockDim.x >> 5);
    const int n = alive.n < 0 ? n_domains : alive.n;
    DomainStart s{};
    if (w < n)
        s = load_start(desc[alive.n < 0 ? w : alive.idx[w]]);
    lists_start(P, close, &s_cur);
    __syncthreads();
    const int cur = s_cur;
    unsigned long long nucleated = 0;
    for (int i = w; i < n; i += nw) {
        const int d = alive.n < 0 ? i : alive.idx[i];
        if (i != w)
            s = load_start(desc[d]);
        start_domain(P, desc[d], s, (unsigned int)d, cur, nucleated);
    }
    if ((threadIdx.x & 31) == 0 && nucleated)
        atomicAdd(&P->stat[0][kStatNucleated], nucleated);
}

__global__ void k_step_begin(PoolState *P) { begin_cycle(P, false, P->desc, P->n_domains, AliveSet{-1, {}}); }

// ---------------------------------------------------------------------------------------------
// One CA cycle after its start (begin_cycle) is three passes over the pool:
//   grow        every record of the current list (kBatch per lane, loads issued first): eligibility
//               and diagonal growth (src/CAupdate.cpp:257-261), drop of finished or
//               re-check-solidified cells, solidification of cells whose liquid mask is empty. A
//               record whose mask must still be built, or whose diagonal reached the cached minimum
//               critical length, goes to the claim queue.
//   claim       one queue entry per thread: the liquid mask from the 26 neighbour types when it is
//               not built yet (nucleated and new-layer cells), the critical-length row (7 aligned
//               16-byte loads) and the claims (src/CAupdate.cpp:320-352); every claim is listed.
//   capture     kCaptureLanes lanes per listed claim: the winner's group captures the cell
//               (src/CAupdate.cpp:353-563), builds the new record's liquid mask and cached minimum
//               critical length, and re-checks the captured cell's active neighbours.
// They run as three kernels per cycle (k_grow, k_claim, k_capture_pass) or, for stretches of
// cycles, inside the persistent cooperative kernel k_cycles with grid-wide barriers between them.
constexpr unsigned int kNeedsClaim = 0xffffffffu; // NaN pattern in ActiveRec::cdl_min
// Launch-shape parameters (template arguments of the passes; the pool's tuner picks among the
// compiled combinations): records per lane in flight in the growth pass, lanes per claim in the
// capture pass.
constexpr int kBatchChoices[2] = {2, 4};
constexpr int kLaneChoices[2] = {4, 8};
constexpr int kErrBarrier = 8;

struct CycleStats {
    unsigned long long listed = 0, grown = 0, dropped = 0, flagged = 0, claims = 0, rows = 0, fresh = 0,
                       captured = 0, rechecks = 0;
};

__device__ void flush_stats(PoolState *P, const CycleStats &st) {
    block_stats(P, st.listed, st.grown, kStatListed, kStatGrown);
    block_stats(P, st.dropped, st.flagged, kStatDropped, kStatFlagged);
    block_stats(P, st.claims, st.rows, kStatClaims, kStatRowReads);
    block_stats(P, st.fresh, st.captured, kStatFresh, kStatCaptured);
    block_stats(P, st.rechecks, 0, kStatRechecks, kStatRechecks);
}

// Growth step of one record with its liquid mask and growth increment loaded. Returns 0: drop
// the record, 1: keep it unchanged (not eligible yet), 2: keep the updated record.
// eff_min: the cached minimum critical length, or the second-smallest one once the minimum's
// neighbour is no longer liquid (both are lower bounds of the current liquid neighbours' lengths).
__device__ __forceinline__ int grow_record(DomainDesc &D, ActiveRec &r, unsigned int m, double inc, bool inc_ok,
                                           float eff_min, CycleStats &st) {
    const unsigned int c = r.cell;
    st.listed++;
    if (D.done || (m & kMaskDead)) {
        // finished domain, or solidified by last cycle's re-check (a retired domain's records point
        // at the placeholder descriptor, which has no fields)
        if (D.dl)
            D.dl[c] = r.dl;
        return 0;
    }
    if (!(D.cycle > r.cts))
        return 1; // cts is INT_MAX outside the window and for LayerID > layer
    st.grown++;
    if (!inc_ok)
        atomicOr(&D.error, kErrGrowthTable);
    const float dl = (float)((double)r.dl + inc);
    r.dl = dl;
    if ((m & kMaskFresh) || dl >= eff_min) {
        r.cdl_min = __uint_as_float(kNeedsClaim);
        st.flagged++;
        return 2;
    }
    if ((m & kDirBits) == 0) {
        // no liquid neighbour: LCount stays 0 (src/CAupdate.cpp:722-725)
        D.ctype[c] = kSolid;
        D.dl[c] = dl;
        return 0;
    }
    return 2;
}

// The descriptor fields a growth step reads for every record, in registers: for the pool's first
// domain they are loaded once per growth pass, for the others per record.
struct GrowView {
    DomainDesc *D;
    const double *growth;
    long long e_cycle; // executed cycles up to the current one
    int cycle, growth_len;
    bool done, jumps, zero_du;
};
__device__ __forceinline__ GrowView grow_view(DomainDesc &D) {
    GrowView v;
    v.D = &D;
    v.growth = D.growth;
    v.cycle = D.cycle;
    v.e_cycle = executed_upto(D, v.cycle);
    v.growth_len = D.growth_len;
    v.done = D.done != 0;
    v.jumps = D.n_jumps > 0;
    v.zero_du = D.zero_du != 0;
    return v;
}

// grow_record with the per-record descriptor fields from a view
__device__ __forceinline__ int grow_record(const GrowView &v, ActiveRec &r, unsigned int m, double inc, bool inc_ok,
                                           float eff_min, CycleStats &st) {
    const unsigned int c = r.cell;
    st.listed++;
    if (v.done || (m & kMaskDead)) {
        if (v.D->dl)
            v.D->dl[c] = r.dl;
        return 0;
    }
    if (!(v.cycle > r.cts))
        return 1;
    st.grown++;
    if (!inc_ok)
        atomicOr(&v.D->error, kErrGrowthTable);
    const float dl = (float)((double)r.dl + inc);
    r.dl = dl;
    if ((m & kMaskFresh) || dl >= eff_min) {
        r.cdl_min = __uint_as_float(kNeedsClaim);
        st.flagged++;
        return 2;
    }
    if ((m & kDirBits) == 0) {
        v.D->ctype[c] = kSolid;
        v.D->dl[c] = dl;
        return 0;
    }
    return 2;
}

__device__ __forceinline__ float effective_min(const ActiveRec &r, unsigned int m, unsigned long long min2) {
    const unsigned int d1 = (unsigned int)(min2 >> 32);
    return (d1 >= 26u || ((m >> d1) & 1u)) ? r.cdl_min : __uint_as_float((unsigned int)min2);
}

// load_growth with the per-record descriptor fields from a view
__device__ __forceinline__ void load_growth(const GrowView &v, const ActiveRec &r, double &inc, bool &ok, bool extras) {
    long long nu = v.e_cycle - (v.jumps ? executed_upto(*v.D, r.cts) : (r.cts <= 0 ? 0ll : (long long)r.cts));
    const double *table = v.growth;
    if (extras) {
        if (v.D->nu_base)
            nu += __ldg(v.D->nu_base + r.cell);
        if (v.D->du_class)
            table += (size_t)__ldg(v.D->du_class + r.cell) * (size_t)v.growth_len;
    }
    if (v.zero_du && v.D->du[r.cell] == 0.0f)
        nu = 0;
    ok = nu >= 0 && nu < v.growth_len;
    inc = (ok && v.cycle > r.cts) ? __ldg(table + nu) : 0.0;
}

__device__ __forceinline__ void load_growth(const DomainDesc &D, const ActiveRec &r, double &inc, bool &ok,
                                            bool extras) {
    // undercooling after the executed updates since the liquidus (src/CAupdate.cpp:236-237), plus
    // those of earlier layers; the growth table of the cell's UndercoolingChange value
    long long nu = executed_upto(D, D.cycle) - executed_upto(D, r.cts);
    const double *table = D.growth;
    if (extras) {
        if (D.nu_base)
            nu += __ldg(D.nu_base + r.cell);
        if (D.du_class)
            table += (size_t)__ldg(D.du_class + r.cell) * (size_t)D.growth_len;
    }
    if (D.zero_du && D.du[r.cell] == 0.0f)
        nu = 0;
    ok = nu >= 0 && nu < D.growth_len;
    inc = (ok && D.cycle > r.cts) ? __ldg(table + nu) : 0.0;
}

// Records the growth pass hands to the claim pass go to a global queue together with the state the
// claim pass needs (list position, cell, domain, liquid-neighbour mask, grown DiagonalLength), so the
// claim pass needs no dependent load before its own round of loads.
// Warp-aggregated reservation of n slots per lane on a global counter (every lane of the warp
// calls). Returns this lane's first slot, or ULLONG_MAX past `cap` (the pool error flag is set).
__device__ __forceinline__ unsigned long long warp_reserve_n(unsigned long long *counter, unsigned long long cap,
                                                             int *error, unsigned int n) {
    const unsigned int lane = threadIdx.x & 31;
    unsigned int incl = n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (unsigned)o)
            incl += v;
    }
    const unsigned int total = __shfl_sync(0xffffffffu, incl, 31);
    unsigned long long base = 0;
    if (lane == 31 && total)
        base = atomicAdd(counter, (unsigned long long)total);
    base = __shfl_sync(0xffffffffu, base, 31);
    if (base + total > cap) {
        if (lane == 31 && total)
            atomicOr(error, kErrListOverflow);
        return ULLONG_MAX;
    }
    return base + incl - n;
}

// Claim work of queue entry k. Returns the directions of the cells it claimed. All loads of the entry
// (critical-length row, neighbour types) go out in one round.
// A record the growth pass flagged for a claim step: its list position, cell, domain, liquid mask
// and grown DiagonalLength.
struct ClaimItem {
    unsigned int pos, cell, dom, mask;
    float dl;
};

__device__ __forceinline__ unsigned int claim_record(PoolState *P, ActiveRec *recs, const ClaimItem &it,
                                                     CycleStats &st, unsigned long long &tombs) {
    const unsigned int i = it.pos, c = it.cell, dom = it.dom;
    unsigned int m = it.mask;
    const float dl = it.dl;
    DomainDesc &D = P->desc[dom];
    const int plane = D.mx * D.my, my = D.my;
    // the 26 critical lengths as 7 aligned 16-byte loads: a row (26 * 4 * c bytes in) starts on a
    // 16-byte boundary for even c and 8 bytes past one for odd c, which read from 8 bytes before it
    // (the previous row's end). The 8 bytes read past an even row lie in the array, or for the last
    // row in the slot's next field array (sub-arrays start on 256-byte boundaries).
    const bool odd = c & 1u;
    const float4 *row = reinterpret_cast<const float4 *>(D.cdl + 26ull * c - (odd ? 2 : 0));
    float f[28];
#pragma unroll
    for (int q = 0; q < 7; q++) {
        const float4 v = __ldcg(row + q);
        f[4 * q] = v.x;
        f[4 * q + 1] = v.y;
        f[4 * q + 2] = v.z;
        f[4 * q + 3] = v.w;
    }
    float cdl[26];
#pragma unroll
    for (int l = 0; l < 26; l++)
        cdl[l] = odd ? f[l + 2] : f[l];
    if (m & kMaskFresh) {
        // liquid neighbours from the 26 neighbour types (src/CAupdate.cpp:320-334); no other thread
        // writes this cell's mask now, captures and nucleations clear bits later. Invalid directions
        // read the cell itself. A cell claimed in this same step (TemporaryUpdate) is still liquid.
        st.fresh++;
        int rx, ry, rz;
        cell_coords(D, c, rx, ry, rz);
        const unsigned int valid = neighbour_mask(D, rx, ry, rz);
        const int8_t *ct = D.ctype + c;
        m = 0;
#pragma unroll
        for (int l = 0; l < 26; l++) {
            const bool v = (valid >> l) & 1u;
            const int8_t nt = __ldcg(ct + (v ? nb_offset(l, plane, my) : 0));
            m |= (v && (nt == kLiquid || nt == kTemporaryUpdate)) ? (1u << l) : 0u;
        }
        P->rstat[P->pending][i] = m | kMaskGrown; // a flagged record was grown this cycle
    }
    if ((m & kDirBits) == 0) {
        // no liquid neighbour: LCount stays 0 (src/CAupdate.cpp:722-725)
        D.ctype[c] = kSolid;
        D.dl[c] = dl;
        recs[i].cell = kTombstone;
        recs[i].cdl_min = 0.0f;
        st.dropped++;
        tombs++;
        return 0;
    }
    st.rows++;
    // Every reached cell is claimed and captured within this cycle, so the cached minimum only
    // covers the liquid neighbours not reached (+inf when none is left).
    float nm = __int_as_float(0x7f800000), nm2 = nm;
    unsigned int d1 = 0xffffffffu;
    unsigned int reach = 0;
#pragma unroll
    for (int l = 0; l < 26; l++) {
        if (m & (1u << l)) {
            if (dl >= cdl[l]) {
                reach |= 1u << l;
            }
            else if (cdl[l] < nm) {
                nm2 = nm;
                nm = cdl[l];
                d1 = l;
            }
            else if (cdl[l] < nm2) {
                nm2 = cdl[l];
            }
        }
    }
    recs[i].cdl_min = nm;
    P->rmin2[P->pending][i] = ((unsigned long long)d1 << 32) | __float_as_uint(nm2);
    if (reach) {
        // claims (src/CAupdate.cpp:336-352): the lowest index wins. Nothing waits for them: every
        // claimant lists its claim and the capture pass keeps the winner's. A claimed cell reads
        // TemporaryUpdate until its capture makes it active, as in the reference's capture
        // (src/CAupdate.cpp:343-352).
        const unsigned long long key = ((unsigned long long)(0xffffffffu - D.epoch) << 32) | (unsigned long long)c;
        unsigned long long *base = D.claim + c;
        for (unsigned int bits = reach; bits; bits &= bits - 1) {
            const int nb = nb_offset(__ffs(bits) - 1, plane, my);
            atomicMin(base + nb, key);
            D.ctype[c + nb] = kTemporaryUpdate;
        }
        st.claims += __popc(reach);
    }
    return reach;
}

// The claim step of global claim-queue entry k.
__device__ __forceinline__ unsigned int claim_entry(PoolState *P, ActiveRec *recs, unsigned long long k,
                                                    CycleStats &st, unsigned long long &tombs) {
    const ClaimItem it{__ldcg(P->qpos + k), __ldcg(P->qcell + k), __ldcg(P->qdom + k), __ldcg(P->qmask + k),
                       __ldcg(P->qdl + k)};
    return claim_record(P, recs, it, st, tombs);
}

// Lists the claims of one record per lane (all lanes of the warp call; reach 0: none) for the
// capture pass, as (domain << 37) | (direction << 32) | claimed cell, in shard `shard`.
__device__ __forceinline__ void list_claims(PoolState *P, unsigned int shard, unsigned int reach, unsigned int dom,
                                            unsigned int cell) {
    const unsigned long long cap = P->shard_cap;
    unsigned long long pos = warp_reserve_n(&P->tcnt_s[shard].v, cap, &P->error, __popc(reach));
    if (reach && pos != ULLONG_MAX) {
        pos += (unsigned long long)shard * cap;
        const DomainDesc &D = P->desc[dom];
        const int plane = D.mx * D.my, my = D.my;
        unsigned long long t = pos;
        for (unsigned int bits = reach; bits; bits &= bits - 1) {
            const int l = __ffs(bits) - 1;
            P->tgt[t++] = ((unsigned long long)dom << 37) | ((unsigned long long)l << 32) |
                          (unsigned int)((long long)cell + nb_offset(l, plane, my));
        }
    }
}

// The flagged records of a block wait in shared memory for the block's own claim step, which starts
// as soon as the block has grown its records (no grid-wide wait between growth and claims). A
// block that flags more than kBlockQueue records in a cycle sends the rest to the global queue,
// whose claim pass then runs after a grid-wide barrier (a flag tells every block).
constexpr int kBlockQueue = 1280;
struct BlockQueue {
    ClaimItem *items;    // kBlockQueue entries in shared memory
    unsigned int *count; // in shared memory; may exceed kBlockQueue (the excess went global)
};

// Puts the flagged records of one growth step into the claim queue (all lanes of the warp call).
template <int kBatch>
__device__ __forceinline__ void queue_flagged(PoolState *P, unsigned int shard, unsigned int nf, unsigned int flagged,
                                              const unsigned long long *idx, const ActiveRec *r,
                                              const unsigned int *dom, const unsigned int *m) {
    unsigned long long k = warp_reserve_n(&P->qcnt_s[shard].v, P->shard_cap, &P->error, nf);
    if (nf && k != ULLONG_MAX) {
        k += (unsigned long long)shard * P->shard_cap;
#pragma unroll
        for (int q = 0; q < kBatch; q++) {
            if (flagged & (1u << q)) {
                P->qpos[k] = (unsigned int)idx[q];
                P->qcell[k] = r[q].cell;
                P->qdom[k] = dom[q];
                P->qmask[k] = m[q];
                P->qdl[k] = r[q].dl;
                k++;
            }
        }
    }
}

// Puts the flagged records of one growth step into the block's queue; those that do not fit go to
// the global queue (all lanes of the warp call). Every slot below kBlockQueue that a warp reserves
// is written in the same step, so the block's claim step reads only this cycle's records.
template <int kBatch>
__device__ __forceinline__ void block_queue_flagged(PoolState *P, BlockQueue bq, unsigned int shard, unsigned int nf,
                                                    unsigned int flagged, const unsigned long long *idx,
                                                    const ActiveRec *r, const unsigned int *dom, const unsigned int *m) {
    const unsigned int lane = threadIdx.x & 31;
    unsigned int incl = nf;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (unsigned)o)
            incl += v;
    }
    const unsigned int total = __shfl_sync(0xffffffffu, incl, 31);
    unsigned int base = 0;
    if (lane == 31 && total)
        base = atomicAdd(bq.count, total);
    base = __shfl_sync(0xffffffffu, base, 31);
    const unsigned int first = base + incl - nf; // this lane's first slot
    unsigned int e = first, n_global = 0;
#pragma unroll
    for (int q = 0; q < kBatch; q++)
        if (flagged & (1u << q)) {
            if (e < (unsigned int)kBlockQueue)
                bq.items[e] = ClaimItem{(unsigned int)idx[q], r[q].cell, dom[q], m[q], r[q].dl};
            else
                n_global++;
            e++;
        }
    if (__any_sync(0xffffffffu, n_global != 0)) {
        unsigned long long k = warp_reserve_n(&P->qcnt_s[shard].v, P->shard_cap, &P->error, n_global);
        if (n_global && k != ULLONG_MAX) {
            k += (unsigned long long)shard * P->shard_cap;
            e = first;
#pragma unroll
            for (int q = 0; q < kBatch; q++)
                if (flagged & (1u << q)) {
                    if (e >= (unsigned int)kBlockQueue) {
                        P->qpos[k] = (unsigned int)idx[q];
                        P->qcell[k] = r[q].cell;
                        P->qdom[k] = dom[q];
                        P->qmask[k] = m[q];
                        P->qdl[k] = r[q].dl;
                        k++;
                    }
                    e++;
                }
        }
    }
}

// The block's claim step over its queue (all threads of the block call, after the block's growth).
__device__ __forceinline__ void block_claims(PoolState *P, BlockQueue bq, unsigned int shard, CycleStats &st,
                                             unsigned long long &tombs) {
    __syncthreads();
    // one store per block: every warp of the grid storing to this flag once its block's queue was
    // full serialised on one L2 slice
    if (threadIdx.x == 0 && *bq.count > (unsigned int)kBlockQueue)
        P->claim_overflow = 1;
    const unsigned int n = min(*bq.count, (unsigned int)kBlockQueue);
    ActiveRec *recs = P->rec[P->pending];
    const unsigned int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (unsigned int k0 = warp * 32; k0 < n; k0 += kBlock) {
        const unsigned int k = k0 + lane;
        unsigned int reach = 0, dom = 0, cell = 0;
        if (k < n) {
            const ClaimItem it = bq.items[k];
            reach = claim_record(P, recs, it, st, tombs);
            dom = it.dom;
            cell = it.cell;
        }
        list_claims(P, shard, reach, dom, cell);
    }
}

// Growth step of a compaction cycle: the survivors are written to the other list (rare; kept out of
// line).
__device__ __noinline__ void compact_pass(PoolState *P, int cur, unsigned long long gw, unsigned long long nw,
                                         unsigned long long n, CycleStats &st, const BlockQueue *bq) {
    const unsigned int lane = threadIdx.x & 31;
    DomainDesc *desc = P->desc;
    const bool extras = P->extras;
    const ActiveRec *in = P->rec[cur];
    const unsigned int *in_dom = P->rdom[cur];
    const unsigned int *in_stat = P->rstat[cur];
    const unsigned long long *in_min2 = P->rmin2[cur];
    const int nxt = cur ^ 1;
    ActiveRec *out = P->rec[nxt];
    unsigned int *out_dom = P->rdom[nxt];
    unsigned int *out_stat = P->rstat[nxt];
    unsigned long long *out_min2 = P->rmin2[nxt];
    const unsigned long long groups = (n + 31) / 32;
    for (unsigned long long g = gw; g < groups; g += nw) {
        unsigned long long i = g * 32 + lane;
        bool keep = false;
        ActiveRec r;
        r.cell = kTombstone;
        unsigned int dom = 0, m = 0;
        unsigned long long mn2 = kNoMin2;
        if (i < n) {
            const int4 v = __ldcg(reinterpret_cast<const int4 *>(in + i));
            r = *reinterpret_cast<const ActiveRec *>(&v);
            dom = __ldcg(in_dom + i);
            m = __ldcg(in_stat + i) & ~kMaskKeep;
            mn2 = __ldcg(in_min2 + i);
            if (r.cell != kTombstone) {
                double inc;
                bool ok;
                load_growth(desc[dom], r, inc, ok, extras);
                const int a = grow_record(desc[dom], r, m, inc, ok, effective_min(r, m, mn2), st);
                keep = a != 0;
                if (a == 2)
                    m |= kMaskGrown;
                if (!keep)
                    st.dropped++;
            }
        }
        const unsigned long long pos = warp_reserve_n(&P->cnt[nxt], P->capacity, &P->error, keep ? 1u : 0u);
        const bool placed = keep && pos != ULLONG_MAX;
        if (placed) {
            out[pos] = r;
            out_dom[pos] = dom;
            out_stat[pos] = m;
            out_min2[pos] = mn2;
            desc[dom].pos[r.cell] = (unsigned int)pos;
        }
        const bool flag = placed && __float_as_uint(r.cdl_min) == kNeedsClaim;
        unsigned long long idx = pos;
        if (bq)
            block_queue_flagged<1>(P, *bq, (unsigned int)(gw % kShards), flag ? 1u : 0u, flag ? 1u : 0u, &idx, &r,
                                   &dom, &m);
        else
            queue_flagged<1>(P, (unsigned int)(gw % kShards), flag ? 1u : 0u, flag ? 1u : 0u, &idx, &r, &dom, &m);
    }
}

// Active records are handed out to warps in groups of 32 consecutive records (one coalesced load),
// group g to warp g % (number of warps of the grid), consecutive warps on different blocks: the
// records appended by the last capture pass, which all need a fresh mask and claims, spread over
// every SM. No block-wide synchronisation.
template <int kBatch, bool kBlockClaims> __device__ void grow_pass(PoolState *P, CycleStats &st, unsigned int hot = 0) {
    const int cur = P->cur;
    const unsigned long long n = P->cnt[cur];
    const unsigned int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned long long nw = (unsigned long long)gridDim.x * (kBlock / 32);
    const unsigned long long gw = (unsigned long long)warp * gridDim.x + blockIdx.x;
    const unsigned int shard = (unsigned int)(gw % kShards);
    __shared__ ClaimItem s_items[kBlockClaims ? kBlockQueue : 1];
    __shared__ unsigned int s_count;
    const BlockQueue bq{s_items, &s_count};
    if (kBlockClaims) {
        if (threadIdx.x == 0)
            s_count = 0;
        __syncthreads();
    }
    if (P->compact) {
        compact_pass(P, cur, gw, nw, n, st, kBlockClaims ? &bq : nullptr);
        if (kBlockClaims) {
            unsigned long long claim_tombs = 0; // a compacted list starts without dropped records
            block_claims(P, bq, shard, st, claim_tombs);
        }
        return;
    }
    ActiveRec *in = P->rec[cur];
    const unsigned int *in_dom = P->rdom[cur];
    unsigned int *in_stat = P->rstat[cur];
    const unsigned long long *in_min2 = P->rmin2[cur];
    DomainDesc *desc = P->desc;
    const bool extras = P->extras;
    unsigned long long tombs = 0;
    const unsigned long long groups = (n + 31) / 32;
    // the growth fields of one domain (the one with the most cells among few) held in registers
    const GrowView v0 = grow_view(desc[hot]);
    // records are updated in place; dropped ones become tombstones
    for (unsigned long long g0 = gw; g0 < groups; g0 += kBatch * nw) {
        ActiveRec r[kBatch];
        unsigned int dom[kBatch], m[kBatch];
        unsigned long long idx[kBatch], mn2[kBatch];
        double inc[kBatch];
        bool ok[kBatch];
#pragma unroll
        for (int q = 0; q < kBatch; q++) {
            idx[q] = (g0 + (unsigned long long)q * nw) * 32 + lane;
            r[q].cell = kTombstone;
            dom[q] = 0;
            m[q] = 0;
            mn2[q] = kNoMin2;
            if (idx[q] < n) {
                // streamed once per cycle: through L2 only
                const int4 v = __ldcg(reinterpret_cast<const int4 *>(in + idx[q]));
                r[q] = *reinterpret_cast<const ActiveRec *>(&v);
                dom[q] = __ldcg(in_dom + idx[q]);
                m[q] = __ldcg(in_stat + idx[q]);
                mn2[q] = __ldcg(in_min2 + idx[q]);
            }
        }
#pragma unroll
        for (int q = 0; q < kBatch; q++) {
            inc[q] = 0.0;
            ok[q] = true;
            if (r[q].cell != kTombstone) {
                if (m[q] & kMaskKeep) {
                    // the neighbour verdict of the previous cycle does not carry over
                    m[q] &= ~kMaskKeep;
                    in_stat[idx[q]] = m[q];
                }
                if (dom[q] == hot)
                    load_growth(v0, r[q], inc[q], ok[q], extras);
                else
                    load_growth(grow_view(desc[dom[q]]), r[q], inc[q], ok[q], extras);
            }
        }
        unsigned int flagged = 0;
#pragma unroll
        for (int q = 0; q < kBatch; q++) {
            if (r[q].cell == kTombstone)
                continue;
            const int a = dom[q] == hot ? grow_record(v0, r[q], m[q], inc[q], ok[q], effective_min(r[q], m[q], mn2[q]), st)
                                      : grow_record(grow_view(desc[dom[q]]), r[q], m[q], inc[q], ok[q],
                                                    effective_min(r[q], m[q], mn2[q]), st);
            if (a == 0) {
                in[idx[q]].cell = kTombstone;
                in[idx[q]].cdl_min = 0.0f;
                st.dropped++;
                tombs++;
            }
            else if (a == 2) {
                *reinterpret_cast<float2 *>(&in[idx[q]].dl) = make_float2(r[q].dl, r[q].cdl_min);
                if (!(m[q] & kMaskGrown)) {
                    m[q] |= kMaskGrown;
                    in_stat[idx[q]] = m[q];
                }
                if (__float_as_uint(r[q].cdl_min) == kNeedsClaim)
                    flagged |= 1u << q;
            }
        }
        if (kBlockClaims)
            block_queue_flagged<kBatch>(P, bq, shard, __popc(flagged), flagged, idx, r, dom, m);
        else
            queue_flagged<kBatch>(P, shard, __popc(flagged), flagged, idx, r, dom, m);
    }
    if (kBlockClaims)
        block_claims(P, bq, shard, st, tombs);
    // dropped records stay as tombstones of the in-place list until the next compaction
#pragma unroll
    for (int o = 16; o; o >>= 1)
        tombs += __shfl_down_sync(0xffffffffu, tombs, o);
    if (lane == 0 && tombs)
        atomicAdd(&P->tomb_s[gw % kShards].v, tombs);
}

// Exclusive prefix of the shard counts in shared memory (all threads of the block call).
__device__ __forceinline__ void shard_prefix(const ShardCounter *cnt, unsigned long long *pre) {
    if (threadIdx.x < 32) {
        const unsigned int lane = threadIdx.x;
        const unsigned long long c = __ldcg(&cnt[lane].v);
        unsigned long long incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            unsigned long long v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (unsigned)o)
                incl += v;
        }
        pre[lane + 1] = incl;
        if (lane == 0)
            pre[0] = 0;
    }
    __syncthreads();
}

// Position in the sharded array of the k-th entry of the shards' concatenation.
__device__ __forceinline__ unsigned long long shard_entry(const unsigned long long *pre, unsigned long long cap,
                                                          unsigned long long k) {
    int lo = 0;
#pragma unroll
    for (int step = 16; step; step >>= 1)
        if (pre[lo + step] <= k)
            lo += step;
    return (unsigned long long)lo * cap + (k - pre[lo]);
}

// One queue entry per thread, consecutive warps on different blocks; every claim is listed.
__device__ void claim_pass(PoolState *P, CycleStats &st) {
    __shared__ unsigned long long s_pre[kShards + 1];
    shard_prefix(P->qcnt_s, s_pre);
    const unsigned long long nq = s_pre[kShards];
    const unsigned long long cap = P->shard_cap;
    ActiveRec *recs = P->rec[P->pending];
    const unsigned int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned long long nw = (unsigned long long)gridDim.x * (kBlock / 32);
    const unsigned long long gw = (unsigned long long)warp * gridDim.x + blockIdx.x;
    unsigned long long tombs = 0;
    for (unsigned long long k0 = gw * 32; k0 < nq; k0 += nw * 32) {
        const unsigned long long k = k0 + lane;
        unsigned int reach = 0, dom = 0, cell = 0;
        if (k < nq) {
            const unsigned long long e = shard_entry(s_pre, cap, k);
            reach = claim_entry(P, recs, e, st, tombs);
            dom = __ldcg(P->qdom + e);
            cell = __ldcg(P->qcell + e);
        }
        list_claims(P, (unsigned int)(gw % kShards), reach, dom, cell);
    }
    if (!P->compact) {
#pragma unroll
        for (int o = 16; o; o >>= 1)
            tombs += __shfl_down_sync(0xffffffffu, tombs, o);
        if (lane == 0 && tombs)
            atomicAdd(&P->tomb_s[gw % kShards].v, tombs);
    }
}

template <int kCaptureLanes> __device__ void capture_pass(PoolState *P, CycleStats &st) {
    __shared__ unsigned long long s_pre[kShards + 1];
    shard_prefix(P->tcnt_s, s_pre);
    const int app = P->pending; // list of the next cycle
    const unsigned long long T = s_pre[kShards];
    const unsigned long long cap = P->shard_cap;
    // records of the cells active at the start of the cycle lie below base; claim j of the cycle
    // gets record slot base + j (a tombstone unless it won), and the count grows by T when the
    // cycle finishes
    const unsigned long long base = P->cnt[app];
    if (base + T > P->capacity) {
        if (threadIdx.x == 0 && blockIdx.x == 0)
            atomicOr(&P->error, kErrListOverflow);
        return;
    }
    DomainDesc *desc = P->desc;
    unsigned long long losers = 0;
    unsigned int *rs = P->rstat[app];
    constexpr int kGroups = 32 / kCaptureLanes;
    constexpr int kPer = (26 + kCaptureLanes - 1) / kCaptureLanes;
    const int lane = threadIdx.x & 31;
    const int grp = lane / kCaptureLanes, sub = lane % kCaptureLanes;
    // consecutive claims on different blocks (spread over all SMs)
    const unsigned long long ngroups = (unsigned long long)gridDim.x * (kBlock / 32) * kGroups;
    const unsigned long long g0 = ((unsigned long long)(threadIdx.x >> 5) * gridDim.x + blockIdx.x) * kGroups + grp;
    for (unsigned long long j = g0; j < T; j += ngroups) {
        const unsigned long long e = __ldcg(P->tgt + shard_entry(s_pre, cap, j));
        const unsigned int t = (unsigned int)e;
        const int l = (int)((e >> 32) & 31u);
        const unsigned int dom = (unsigned int)(e >> 37);
        DomainDesc &D = desc[dom];
        const int plane = D.mx * D.my, my = D.my;
        const unsigned int c = (unsigned int)((long long)t - nb_offset(l, plane, my)); // the claimant
        // Every load of the capture and of the re-checks goes out in one round; only the group of
        // the winning claim (the lowest claimant index) continues. Lane `sub` takes the neighbour
        // slots sub, sub + kCaptureLanes, ... (slot_dir): a load instruction's lanes read
        // neighbours in few rows of three consecutive cells.
        const unsigned long long key = __ldcg(D.claim + t);
        const int cts_t = __ldg(D.cts_run + t);
        const int h = __ldcg(D.gid + c);
        const float docx = __ldcg(D.doc + 3ull * c + 0), docy = __ldcg(D.doc + 3ull * c + 1),
                    docz = __ldcg(D.doc + 3ull * c + 2);
        int tx, ty, tz;
        cell_coords(D, t, tx, ty, tz);
        const unsigned int valid = neighbour_mask(D, tx, ty, tz);
        unsigned int a[kPer], p[kPer], old[kPer];
        int8_t ct[kPer];
        bool act[kPer];
#pragma unroll
        for (int k = 0; k < kPer; k++) {
            const int ln = slot_dir(sub + k * kCaptureLanes);
            act[k] = ln < 26 && (valid & (1u << ln));
            a[k] = (unsigned int)((long long)t + (act[k] ? nb_offset(ln, plane, my) : 0));
            ct[k] = __ldcg(D.ctype + a[k]);
            p[k] = __ldcg(D.pos + a[k]);
        }
        if ((unsigned int)key != c) {
            // a lower-index claimant captures t; this claim's slot stays a dropped record
            if (sub == 0) {
                P->rec[app][base + j].cell = kTombstone;
                P->rec[app][base + j].cdl_min = 0.0f;
                losers++;
            }
            continue;
        }
        const unsigned int w = c;
        // The captured cell's liquid-neighbour mask, as its first claim step would build it from the
        // neighbour types at the start of a later cycle: the neighbours still liquid (a neighbour
        // claimed in this cycle reads TemporaryUpdate, or active once captured). Later captures and
        // nucleations clear bits of it as of every other record's (it lies below later cycles' base).
        unsigned int liq = 0;
#pragma unroll
        for (int k = 0; k < kPer; k++)
            if (act[k] && ct[k] == kLiquid)
                liq |= 1u << slot_dir(sub + k * kCaptureLanes);
        {
            const unsigned int group = (kCaptureLanes == 32 ? 0xffffffffu : ((1u << kCaptureLanes) - 1u))
                                       << (grp * kCaptureLanes);
#pragma unroll
            for (int o = kCaptureLanes / 2; o; o >>= 1)
                liq |= __shfl_xor_sync(group, liq, o);
        }
        // Serial order (src/CAupdate.cpp:333-334, 722-725): active cell a saw the captured cell t
        // as liquid iff t's capturer w does not precede a. a keeps a liquid neighbour iff it has an
        // unclaimed one (a set mask bit that nobody clears) or a claimed one with w >= a. Every
        // claimed liquid neighbour clears its own bit exactly once, so the update that clears the
        // last direction bit sees the final verdict: KEEP is always set before the clear of the
        // same update, and an update's two atomics reach the word in program order. Only records of
        // cells active at the start of the cycle (positions below base) take part: a neighbour
        // captured in this same cycle reads as liquid, or has no record below base.
#pragma unroll
        for (int k = 0; k < kPer; k++)
            act[k] = act[k] && ct[k] == kActive && p[k] < base;
#pragma unroll
        for (int k = 0; k < kPer; k++)
            if (act[k] && w >= a[k])
                atomicOr(rs + p[k], kMaskKeep);
#pragma unroll
        for (int k = 0; k < kPer; k++) {
            old[k] = 0;
            if (act[k])
                old[k] = atomicAnd(rs + p[k], ~(1u << nb_opp(slot_dir(sub + k * kCaptureLanes))));
        }
        // The new record's cached minimum critical length over its liquid neighbours, with its
        // direction and the second-smallest (the state a claim step leaves), so that its first claim
        // step runs only once its DiagonalLength reaches a liquid neighbour.
        float mn = __int_as_float(0x7f800000), mn2 = mn;
        unsigned int d1 = 0xffffffffu;
        const float new_dl =
            capture_cell<kCaptureLanes>(D, c, t, l, sub, h, docx, docy, docz, liq, mn, d1, mn2);
        {
            const unsigned int group = (kCaptureLanes == 32 ? 0xffffffffu : ((1u << kCaptureLanes) - 1u))
                                       << (grp * kCaptureLanes);
#pragma unroll
            for (int o = kCaptureLanes / 2; o; o >>= 1) {
                const float omn = __shfl_xor_sync(group, mn, o), omn2 = __shfl_xor_sync(group, mn2, o);
                const unsigned int od1 = __shfl_xor_sync(group, d1, o);
                if (omn < mn || (omn == mn && od1 < d1)) {
                    mn2 = fminf(omn2, mn);
                    mn = omn;
                    d1 = od1;
                }
                else {
                    mn2 = fminf(mn2, omn);
                }
            }
        }
        if (sub == 0) {
            ActiveRec r;
            r.cell = t;
            r.dl = new_dl;
            r.cdl_min = mn;
            r.cts = cts_t;
            P->rec[app][base + j] = r;
            P->rdom[app][base + j] = dom;
            rs[base + j] = liq;
            P->rmin2[app][base + j] = ((unsigned long long)d1 << 32) | __float_as_uint(mn2);
            D.pos[t] = (unsigned int)(base + j);
            // read as active by the growth pass of the next cycle, after the octahedron is written
            D.ctype[t] = kActive;
            atomicAdd((unsigned long long *)&D.liquid_shard[(blockIdx.x + j) & (kLiquidShards - 1)],
                      (unsigned long long)(-1ll));
            st.captured++;
        }
#pragma unroll
        for (int k = 0; k < kPer; k++) {
            if (!act[k])
                continue;
            const unsigned int bit = 1u << nb_opp(slot_dir(sub + k * kCaptureLanes));
            if ((old[k] & (kMaskFresh | kMaskDead)) || (old[k] & kDirBits) != bit || (old[k] & kMaskKeep))
                continue;
            // a lost its last liquid neighbour; it solidifies if it was grown this cycle (cycle >
            // its CritTimeStep, src/CAupdate.cpp:257-261)
            if (old[k] & kMaskGrown) {
                st.rechecks++;
                D.ctype[a[k]] = kSolid;
                atomicOr(rs + p[k], kMaskDead);
            }
        }
    }
    // every lane reaches this point
#pragma unroll
    for (int o = 16; o; o >>= 1)
        losers += __shfl_down_sync(0xffffffffu, losers, o);
    if (lane == 0 && losers)
        atomicAdd(&P->tomb_s[(blockIdx.x + threadIdx.x) % kShards].v, losers);
}

// End of a cycle: the record slots of this cycle's claims join the list.
__device__ void finish_capture(PoolState *P) {
    if (threadIdx.x < 32) {
        unsigned long long T = __ldcg(&P->tcnt_s[threadIdx.x].v);
#pragma unroll
        for (int o = 16; o; o >>= 1)
            T += __shfl_down_sync(0xffffffffu, T, o);
        if (threadIdx.x == 0) {
            const int app = P->pending;
            if (P->cnt[app] + T <= P->capacity)
                P->cnt[app] += T;
        }
    }
    __syncthreads();
}

template <int kBatch> __global__ void __launch_bounds__(kBlock) k_grow(PoolState *P) {
    CycleStats st;
    grow_pass<kBatch, false>(P, st);
    flush_stats(P, st);
}

__global__ void __launch_bounds__(kBlock) k_claim(PoolState *P) {
    CycleStats st;
    claim_pass(P, st);
    flush_stats(P, st);
}

// Capture pass as its own kernel; the last block to finish closes the cycle and, with kBegin,
// starts the next one.
template <bool kBegin, int kLanes> __global__ void __launch_bounds__(kBlock) k_capture_pass(PoolState *P) {
    CycleStats st;
    capture_pass<kLanes>(P, st);
    flush_stats(P, st);
    __shared__ int s_last;
    __threadfence(); // this block's writes are visible device-wide before it is counted
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int prev = atomicAdd(&P->blocks_done, 1u);
        s_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (s_last) {
        __threadfence();
        if (threadIdx.x == 0)
            P->blocks_done = 0;
        if (kBegin)
            begin_cycle(P, true, P->desc, P->n_domains, AliveSet{-1, {}});
        else
            finish_capture(P);
    }
}

// ---------------------------------------------------------------------------------------------
// Grid-wide meeting point of the persistent kernel (all blocks co-resident: cooperative launch).
// Arrival is an acq_rel atomic on a counter, release an st.release of the next generation; the
// last block to arrive runs `serial` with the whole block before it releases the others. Every
// wait is bounded: after kMeetTimeoutNs (or kMeetSpinCap polls) the block sets kErrBarrier and
// the kernel ends.
constexpr unsigned long long kMeetTimeoutNs = 1000000000ull;
constexpr unsigned int kMeetSpinCap = 1u << 26;

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int *p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned int atom_add_acq_rel_u32(unsigned int *p, unsigned int v) {
    unsigned int old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
__device__ __forceinline__ void st_release_u32(unsigned int *p, unsigned int v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// With P->timeline set, meeting point `tag` records its first arrival, last arrival and release.
template <class F> __device__ bool grid_meet(PoolState *P, int tag, F &&serial) {
    __shared__ unsigned int s_gen;
    __shared__ int s_state; // 0: released, 1: last to arrive, 2: gave up waiting
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned int gen = ld_acquire_u32(&P->bar_gen);
        const unsigned int prev = atom_add_acq_rel_u32(&P->bar_count, 1u);
        unsigned long long *tl = tag >= 0 ? P->timeline : nullptr;
        if (tl && prev == 0)
            tl[3 * tag + 0] = global_ns();
        int state = 0;
        if (prev == gridDim.x - 1) {
            state = 1;
            if (tl)
                tl[3 * tag + 1] = global_ns();
        }
        else {
            const unsigned long long t0 = global_ns();
            unsigned int it = 0;
            while (ld_acquire_u32(&P->bar_gen) == gen) {
                ++it;
                if (it >= kMeetSpinCap || ((it & 255u) == 0 && global_ns() - t0 > kMeetTimeoutNs)) {
                    atomicOr(&P->error, kErrBarrier);
                    state = 2;
                    break;
                }
                __nanosleep(32);
            }
        }
        s_gen = gen;
        s_state = state;
    }
    __syncthreads();
    const int state = s_state;
    if (state == 1) {
        serial();
        __syncthreads();
        if (threadIdx.x == 0) {
            if (P->timeline && tag >= 0)
                P->timeline[3 * tag + 2] = global_ns();
            P->bar_count = 0;
            st_release_u32(&P->bar_gen, s_gen + 1u);
        }
    }
    return state != 2;
}

// n_cycles complete CA cycles (start, grow/claim, capture) in one cooperative launch.
template <int kLanes, int kBatch>
__global__ void __launch_bounds__(kBlock, 1) k_cycles(PoolState *P, int n_cycles, AliveSet alive) {
    CycleStats st;
    // with many running domains, their per-cycle start (termination, nucleation) runs across the
    // grid (the descriptors and their number change only between launches); with a few, one block
    // starts them, and the first one's growth fields stay in registers
    DomainDesc *const desc = P->desc;
    const int n_domains = P->n_domains;
    const bool spread = alive.n < 0 && n_domains > kSerialDomains;
    const unsigned int hot = alive.n > 0 ? (unsigned int)alive.idx[0] : 0u;
    const int gwarp = (threadIdx.x >> 5) * gridDim.x + blockIdx.x, nwarp = gridDim.x * (kBlock / 32);
    bool ok = grid_meet(P, 0, [&] {
        if (spread)
            begin_lists(P, false);
        else
            begin_cycle(P, false, desc, n_domains, alive);
    });
    if (ok && spread) {
        begin_domains(P, desc, n_domains, gwarp, nwarp);
        ok = grid_meet(P, -1, [] {});
    }
    for (int c = 0; ok && c < n_cycles; c++) {
        // growth with each block's claims right after its own growth; the global claim pass only
        // when some block's queue overflowed this cycle (the same answer for every block)
        grow_pass<kBatch, true>(P, st, hot);
        ok = grid_meet(P, 3 * c + 1, [] {});
        if (!ok)
            break;
        if (__ldcg(&P->claim_overflow)) {
            claim_pass(P, st);
            ok = grid_meet(P, 3 * c + 2, [] {});
            if (!ok)
                break;
        }
        capture_pass<kLanes>(P, st);
        const bool more = c + 1 < n_cycles;
        ok = grid_meet(P, 3 * c + 3, [&] {
            if (!more)
                finish_capture(P);
            else if (spread)
                begin_lists(P, true);
            else
                begin_cycle(P, true, desc, n_domains, alive);
        });
        if (ok && more && spread) {
            begin_domains(P, desc, n_domains, gwarp, nwarp);
            ok = grid_meet(P, -1, [] {});
        }
    }
    flush_stats(P, st);
}

// The bounded wait of the meeting point taken to its limit: a cooperative launch of two blocks in
// which block 0 leaves without arriving, so block 1's wait can only end by its time limit (it sets
// kErrBarrier and returns, and the context stays usable).
__global__ void __launch_bounds__(kBlock) k_meet_probe(PoolState *P) {
    if (blockIdx.x == 0)
        return;
    grid_meet(P, -1, [] {});
}

// Compiled launch shapes: {capture lanes, growth batch} for kLaneChoices x kBatchChoices.
struct StepKernels {
    const void *cycles;
    void (*grow)(PoolState *);
    void (*capture_begin)(PoolState *);
    void (*capture_end)(PoolState *);
};
template <int kL, int kB> StepKernels step_kernels() {
    return {(const void *)k_cycles<kL, kB>, k_grow<kB>, k_capture_pass<true, kL>, k_capture_pass<false, kL>};
}
static_assert(kStepVariants == 4, "two lane widths x two batch depths");
const StepKernels kStepKernel[kStepVariants] = {
    step_kernels<kLaneChoices[0], kBatchChoices[0]>(), step_kernels<kLaneChoices[0], kBatchChoices[1]>(),
    step_kernels<kLaneChoices[1], kBatchChoices[0]>(), step_kernels<kLaneChoices[1], kBatchChoices[1]>()};

// ---------------------------------------------------------------------------------------------
// Census of src/CAupdate.cpp:738-808 for one domain and its current layer; the smallest
// CritTimeStep is taken over liquid cells of the layer inside the active window. Each thread reads
// 16 cells per step with 16-byte loads (the field arrays start on 256-byte boundaries); the tail of
// fewer than 16 cells is read cell by cell.
struct CensusCount {
    unsigned int superheated = 0, undercooled = 0, active = 0, solid = 0, remaining = 0;
    unsigned long long mn = ULLONG_MAX;
    __device__ __forceinline__ void cell(long long c, int t, int ly, int cts, int cycle, int layer, long long w_lo,
                                         long long w_hi) {
        if (ly == layer) {
            if (t == kLiquid) {
                if (cts > cycle)
                    superheated++;
                else
                    undercooled++;
                const unsigned long long u = (unsigned long long)(long long)cts;
                if (c >= w_lo && c < w_hi && u < mn)
                    mn = u;
            }
            else if (t == kActive)
                active++;
            else if (t == kSolid)
                solid++;
        }
        else if (t == kLiquid) {
            remaining++;
        }
    }
};

__global__ void __launch_bounds__(256) k_census(const DomainDesc *Dp, Census *out) {
    const DomainDesc &D = *Dp;
    const int8_t *ctype = D.ctype, *lay = D.layer;
    const int32_t *ctsp = D.cts;
    const long long N = D.domain_size;
    const int cycle = D.cycle, layer = D.layer_no;
    const long long plane = (long long)D.mx * D.my;
    const long long w_lo = plane * D.z_lo, w_hi = plane * D.z_end;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    CensusCount k;
    const long long n16 = N / 16;
    for (long long q = tid; q < n16; q += stride) {
        const int4 t16 = __ldcs(reinterpret_cast<const int4 *>(ctype) + q);
        const int4 l16 = __ldcs(reinterpret_cast<const int4 *>(lay) + q);
        int4 c4[4];
#pragma unroll
        for (int u = 0; u < 4; u++)
            c4[u] = __ldcs(reinterpret_cast<const int4 *>(ctsp) + 4 * q + u);
        const int tw[4] = {t16.x, t16.y, t16.z, t16.w}, lw[4] = {l16.x, l16.y, l16.z, l16.w};
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int cv[4] = {c4[u].x, c4[u].y, c4[u].z, c4[u].w};
#pragma unroll
            for (int b = 0; b < 4; b++) {
                const int t = (int)(int8_t)(tw[u] >> (8 * b)), ly = (int)(int8_t)(lw[u] >> (8 * b));
                k.cell(16 * q + 4 * u + b, t, ly, cv[b], cycle, layer, w_lo, w_hi);
            }
        }
    }
    for (long long c = 16 * n16 + tid; c < N; c += stride)
        k.cell(c, ctype[c], lay[c], ctsp[c], cycle, layer, w_lo, w_hi);
    const unsigned int counts[5] = {k.superheated, k.undercooled, k.active, k.solid, k.remaining};
#pragma unroll
    for (int q = 0; q < 5; q++) {
        unsigned long long v = counts[q];
        for (int o = 16; o; o >>= 1)
            v += __shfl_down_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0 && v)
            atomicAdd((unsigned long long *)out + q, v);
    }
    unsigned long long mn = k.mn;
    for (int o = 16; o; o >>= 1) {
        unsigned long long v = __shfl_down_sync(0xffffffffu, mn, o);
        mn = v < mn ? v : mn;
    }
    if ((threadIdx.x & 31) == 0)
        atomicMin(&out->next_cts, mn);
}

// Voronoi baseplate (src/CAinitialize.cpp:1646-1677): nearest seed by float distance, the first
// seed in draw order wins ties.
__global__ void k_voronoi(DomainDesc *Dp, const int32_t *seeds, int nseeds, float init_min) {
    extern __shared__ int s_seed[];
    const DomainDesc &D = *Dp;
    long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    bool mine = c < D.domain_size && D.gid[c] == kVoronoiPending;
    int gx = 0, gy = 0, k = 0;
    if (mine) {
        int plane = D.mx * D.my;
        k = (int)(c / plane);
        int rem = (int)(c - (long long)k * plane);
        gx = rem / D.my + D.xoff;
        gy = rem % D.my + D.yoff;
    }
    float best = init_min;
    int best_i = -1;
    for (int base = 0; base < nseeds; base += 1024) {
        int cnt = min(1024, nseeds - base);
        __syncthreads();
        for (int q = threadIdx.x; q < 3 * cnt; q += blockDim.x)
            s_seed[q] = seeds[3 * base + q];
        __syncthreads();
        if (mine) {
            for (int q = 0; q < cnt; q++) {
                float dx = (float)(abs(s_seed[3 * q] - gx));
                float dy = (float)(abs(s_seed[3 * q + 1] - gy));
                float dz = (float)(abs(s_seed[3 * q + 2] - k));
                float dist = sqrtf(dx * dx + dy * dy + dz * dz);
                if (dist < best) {
                    best_i = base + q;
                    best = dist;
                }
            }
        }
    }
    if (mine)
        D.gid[c] = best_i + 1;
}

// Active cells of the active window: fresh octahedra and their records. At admission these are
// the initially active cells (src/CAinitialize.cpp:1929-2044); at the start of a later layer, the
// active cells of the moved window (LayerSetup, src/CAinitialize.cpp:2840-2982).
__global__ void k_init_active(PoolState *P, int dom, int list_slot) {
    if (list_slot < 0)
        list_slot = P->pending; // the list the next cycle consumes
    DomainDesc &D = P->desc[dom];
    long long plane = (long long)D.mx * D.my;
    long long lo = plane, hi = plane * (D.nz - 1);
    if (lo < plane * D.z_lo)
        lo = plane * D.z_lo;
    if (hi > plane * D.z_end)
        hi = plane * D.z_end;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long c0 = lo + (long long)blockIdx.x * blockDim.x; c0 < hi; c0 += stride) {
        long long c = c0 + threadIdx.x;
        bool act = c < hi && D.ctype[c] == kActive;
        if (act)
            make_fresh_octahedron(D, (unsigned int)c);
        bool listed = act;
        unsigned long long pos = block_reserve(P, list_slot, listed ? 1u : 0u);
        if (listed && pos != ULLONG_MAX) {
            ActiveRec r;
            r.cell = (unsigned int)c;
            r.dl = 0.01f;
            r.cdl_min = 0.0f;
            r.cts = D.cts_run[c];
            P->rec[list_slot][pos] = r;
            P->rdom[list_slot][pos] = (unsigned int)dom;
            P->rstat[list_slot][pos] = kMaskFresh;
            P->rmin2[list_slot][pos] = kNoMin2;
            D.pos[c] = (unsigned int)pos;
        }
    }
}

// Re-labels every record of one domain in the list the next cycle consumes with the pool's
// always-finished placeholder domain (used when a slot is retired, before the slot is reused).
__global__ void k_drop_domain(PoolState *P, unsigned int dom, unsigned int placeholder) {
    const int nxt = P->pending;
    unsigned long long n = P->cnt[nxt];
    unsigned int *d = P->rdom[nxt];
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x)
        if (d[i] == dom)
            d[i] = placeholder;
}

// Diagonal lengths held in the pending records back to the per-cell arrays.
__global__ void k_flush_records(PoolState *P) {
    const int nxt = P->pending;
    unsigned long long n = P->cnt[nxt];
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const ActiveRec r = P->rec[nxt][i];
        if (r.cell == kTombstone)
            continue; // a dropped record's other fields are not kept up to date
        const DomainDesc &D = P->desc[P->rdom[nxt][i]];
        if (D.dl)
            D.dl[r.cell] = r.dl;
    }
}

// ---------------------------------------------------------------------------------------------
// Cell fields of a type-C problem made on the device (src/CAinitialize.cpp:1025-1055, 1460-1529,
// 1834-2247): walls on the ghost ring and the bottom and top planes, liquid elsewhere, the plane's
// CritTimeStep, LayerID 0, one UndercoolingChange value; then the substrate seeds (active, GrainID
// rank + 1) and the nuclei (GrainID -(rank + 1), in index order).
__global__ void k_fill_directional(int8_t *ctype, int32_t *gid, int32_t *cts, int8_t *layer, float *du, long long n,
                                   int mx, int my, int nz, const int32_t *plane_cts, float du_value) {
    const long long plane = (long long)mx * my;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(c / plane);
        const int rem = (int)(c - (long long)k * plane);
        const int i = rem / my, j = rem - (rem / my) * my;
        const bool wall = i == 0 || i == mx - 1 || j == 0 || j == my - 1 || k == 0 || k == nz - 1;
        ctype[c] = wall ? kWall : kLiquid;
        gid[c] = 0;
        cts[c] = __ldg(plane_cts + k);
        layer[c] = 0;
        du[c] = du_value;
    }
}

__global__ void k_widen_types(const int8_t *ctype, int32_t *out, long long n) {
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
        out[c] = ctype[c];
}

__global__ void k_scatter_seeds(int8_t *ctype, int32_t *gid, const long long *active, long long n_active,
                                const int32_t *nuclei, long long n_nuclei) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n_active) {
        ctype[active[q]] = kActive;
        gid[active[q]] = (int32_t)(q + 1);
    }
    else if (q < n_active + n_nuclei) {
        const long long r = q - n_active;
        gid[nuclei[r]] = -(int32_t)(r + 1);
    }
}

// ---------------------------------------------------------------------------------------------
// Layer change of a multilayer domain (src/runCA.cpp:344-411).

// Undercooling updates of the ending layer, carried into the next: every liquid or active cell of
// the window whose LayerID <= layer had UndercoolingCurrent += UndercoolingChange once per executed
// cycle past its CritTimeStep (src/CAupdate.cpp:228-237).
__global__ void k_layer_base(const DomainDesc *Dp) {
    const DomainDesc &D = *Dp;
    const long long plane = (long long)D.mx * D.my;
    const long long hi = plane * D.z_end;
    const long long end = executed_upto(D, D.cycle);
    for (long long c = plane * D.z_lo + (long long)blockIdx.x * blockDim.x + threadIdx.x; c < hi;
         c += (long long)gridDim.x * blockDim.x) {
        const int t = D.ctype[c];
        if ((t != kLiquid && t != kActive) || D.layer[c] > D.layer_no)
            continue;
        const long long n = end - executed_upto(D, D.cts[c]);
        if (n > 0)
            D.nu_base[c] += (int32_t)n;
    }
}

// DomainShiftAndResize's two reductions (src/CAinitialize.cpp:2781-2812): the lowest z of an
// active cell and the highest z of a cell of the next layer. out = {INT_MAX, INT_MIN} on entry.
__global__ void k_layer_bounds(const DomainDesc *Dp, int next_layer, int *out) {
    const DomainDesc &D = *Dp;
    const long long plane = (long long)D.mx * D.my;
    int zmin = INT_MAX, zmax = INT_MIN;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < D.domain_size;
         c += (long long)gridDim.x * blockDim.x) {
        const int z = (int)(c / plane);
        if (D.ctype[c] == kActive)
            zmin = min(zmin, z);
        if (D.layer[c] == next_layer)
            zmax = max(zmax, z);
    }
    for (int o = 16; o; o >>= 1) {
        zmin = min(zmin, __shfl_down_sync(0xffffffffu, zmin, o));
        zmax = max(zmax, __shfl_down_sync(0xffffffffu, zmax, o));
    }
    if ((threadIdx.x & 31) == 0) {
        if (zmin != INT_MAX)
            atomicMin(out, zmin);
        if (zmax != INT_MIN)
            atomicMax(out + 1, zmax);
    }
}

// The CritTimeStep the step uses this layer: the cell's own inside the window for LayerID <= layer,
// INT_MAX elsewhere (src/CAupdate.cpp:218-231 visits only window cells, and grows those with
// LayerID <= layernumber).
__global__ void k_layer_gate(const DomainDesc *Dp) {
    const DomainDesc &D = *Dp;
    const long long plane = (long long)D.mx * D.my;
    const long long lo = plane * D.z_lo, hi = plane * D.z_end;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < D.domain_size;
         c += (long long)gridDim.x * blockDim.x)
        D.cts_run[c] = (c >= lo && c < hi && D.layer[c] <= D.layer_no) ? D.cts[c] : INT_MAX;
}

// ---------------------------------------------------------------------------------------------
// Pool runtime

namespace {
inline cudaStream_t S(void *s) { return (cudaStream_t)s; }
template <class T> T *dalloc(size_t n, std::vector<void *> &allocs, size_t &bytes) {
    void *p = nullptr;
    size_t b = std::max<size_t>(n * sizeof(T), 16);
    CUDA_OK(cudaMalloc(&p, b));
    allocs.push_back(p);
    bytes += b;
    return (T *)p;
}

// true when p is page-locked (or registered) host memory that a copy engine writes directly
bool host_pinned(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// Moves one staged piece into the caller's buffer on several host threads: len bytes, or with
// widen len int8 values sign-extended to int32.
void stage_move(char *dst, const char *src, size_t len, bool widen) {
    constexpr size_t kPerThread = size_t(1) << 20;
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t nt = std::max<size_t>(1, std::min<size_t>({(size_t)hw, 8, len / kPerThread}));
    auto part = [&](size_t t) {
        const size_t lo = len * t / nt, hi = len * (t + 1) / nt;
        if (widen) {
            int32_t *o = (int32_t *)dst;
            const int8_t *i = (const int8_t *)src;
            for (size_t k = lo; k < hi; k++)
                o[k] = i[k];
        } else {
            std::memcpy(dst + lo, src + lo, hi - lo);
        }
    };
    std::vector<std::thread> workers;
    for (size_t t = 1; t < nt; t++)
        workers.emplace_back(part, t);
    part(0);
    for (auto &w : workers)
        w.join();
}
} // namespace

void Pool::to_host(const std::vector<HostCopy> &copies, void *stream) {
    constexpr size_t kStageBytes = size_t(32) << 20;
    cudaStream_t st = S(stream);
    // page-locked destinations take their DMA as they are; the rest go through the staging pieces
    struct Piece {
        char *dst;
        const char *src;
        size_t len;
        bool widen;
    };
    std::vector<Piece> pieces;
    for (const HostCopy &c : copies) {
        if (!c.dst || !c.bytes)
            continue;
        if (!c.widen && host_pinned(c.dst)) {
            CUDA_OK(cudaMemcpyAsync(c.dst, c.src, c.bytes, cudaMemcpyDeviceToHost, st));
            continue;
        }
        for (size_t off = 0; off < c.bytes; off += kStageBytes)
            pieces.push_back({(char *)c.dst + (c.widen ? 4 * off : off), (const char *)c.src + off,
                              std::min(kStageBytes, c.bytes - off), c.widen});
    }
    if (pieces.empty())
        return;
    if (!stage_[0]) {
        for (int b = 0; b < 2; b++) {
            CUDA_OK(cudaMallocHost(&stage_[b], kStageBytes));
            cudaEvent_t e;
            CUDA_OK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            stage_ev_[b] = e;
        }
    }
    // two pieces in flight: the DMA of piece k+1 runs while the host threads move piece k out
    auto issue = [&](size_t k) {
        CUDA_OK(cudaMemcpyAsync(stage_[k & 1], pieces[k].src, pieces[k].len, cudaMemcpyDeviceToHost, st));
        CUDA_OK(cudaEventRecord((cudaEvent_t)stage_ev_[k & 1], st));
    };
    issue(0);
    for (size_t k = 0; k < pieces.size(); k++) {
        if (k + 1 < pieces.size())
            issue(k + 1);
        CUDA_OK(cudaEventSynchronize((cudaEvent_t)stage_ev_[k & 1]));
        stage_move(pieces[k].dst, (const char *)stage_[k & 1], pieces[k].len, pieces[k].widen);
    }
}

void pin_problem(Problem &p) {
    auto reg = [](void *ptr, size_t bytes) {
        if (bytes == 0)
            return;
        cudaError_t e = cudaHostRegister(ptr, bytes, cudaHostRegisterDefault);
        if (e != cudaSuccess && e != cudaErrorHostMemoryAlreadyRegistered)
            throw DeviceError(std::string("CUDA error ") + cudaGetErrorString(e) + " at cudaHostRegister");
        cudaGetLastError();
    };
    reg(p.cell_type.data(), p.cell_type.size());
    reg(p.grain_id.data(), p.grain_id.size() * 4);
    reg(p.cts.data(), p.cts.size() * 4);
    reg(p.layer_id.data(), p.layer_id.size());
    reg(p.du.data(), p.du.size() * 4);
    p.pinned = true;
}

void unpin_problem(Problem &p) {
    if (!p.pinned)
        return;
    for (void *ptr : {(void *)p.cell_type.data(), (void *)p.grain_id.data(), (void *)p.cts.data(),
                      (void *)p.layer_id.data(), (void *)p.du.data()})
        if (ptr)
            cudaHostUnregister(ptr);
    cudaGetLastError();
    p.pinned = false;
}

// Multilayer problems keep the per-cell octahedron state for the whole domain (the active window
// moves up layer by layer), plus the per-layer CritTimeStep gate and the undercooling carried over.
static size_t octahedron_cells(const Problem &p) {
    return p.cfg.number_of_layers > 1 ? (size_t)p.g.domain_size : (size_t)p.g.active_size;
}

size_t Pool::slot_bytes(const Problem &p) {
    size_t N = (size_t)p.g.domain_size, A = octahedron_cells(p);
    size_t multilayer = p.cfg.number_of_layers > 1 ? N * 8 : 0;
    size_t classes = p.du_values.size() > 1 ? N * 2 : 0;
    return N * (1 + 4 + 4 + 1 + 4) + A * (4 + 12 + 104 + 8 + 4) + multilayer + classes + p.nuclei_loc.size() * 8 +
           64 * 1024;
}

Pool::Pool(int device, size_t budget_bytes, unsigned long long list_capacity)
    : device_(device), budget_(budget_bytes) {
    CUDA_OK(cudaSetDevice(device));
    cudaDeviceProp prop;
    CUDA_OK(cudaGetDeviceProperties(&prop, device));
    num_sms_ = prop.multiProcessorCount;
    cudaStream_t s;
    CUDA_OK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    stream_ = s;
    // the device's edge masks (edge_mask) are the reference's ItList cases
    int it[9][26], lens[9];
    build_itlist(it, lens);
    for (int b = 0; b < 9; b++) {
        unsigned int m = 0, want = (1u << 26) - 1u;
        for (int q = 0; q < lens[b]; q++)
            m |= 1u << it[b][q];
        if (b == 1 || b == 5 || b == 6)
            want &= ~kDirYM;
        if (b == 2 || b == 7 || b == 8)
            want &= ~kDirYP;
        if (b == 3 || b == 5 || b == 7)
            want &= ~kDirXM;
        if (b == 4 || b == 6 || b == 8)
            want &= ~kDirXP;
        if (m != want)
            throw std::logic_error("edge masks differ from ItList");
    }
    max_domains_ = 8192;
    // list positions are 32-bit in the passes' block-local queues
    if (list_capacity > 0xffffffffull)
        throw Unsupported("list capacity above 2^32 - 1 records");
    capacity_ = std::max<unsigned long long>(list_capacity, 1024);
    int coop = 0;
    CUDA_OK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device));
    if (!coop)
        throw DeviceError("device does not support cooperative launches");
    int b = 0;
    for (int v = 0; v < kStepVariants; v++) {
        CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kStepKernel[v].cycles, kBlock, 0));
        if (b < 1)
            throw DeviceError("persistent kernel does not fit on an SM");
        grid_cycles_[v] = num_sms_ * b;
        CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, (const void *)kStepKernel[v].grow, kBlock, 0));
        grid_grow_[v] = num_sms_ * std::max(b, 1);
        CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, (const void *)kStepKernel[v].capture_end, kBlock, 0));
        grid_capture_[v] = num_sms_ * std::max(b, 1);
    }
    CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_claim, kBlock, 0));
    grid_claim_ = num_sms_ * std::max(b, 1);
    if (const char *m = std::getenv("EXACA_STEP_MODE"))
        step_mode_ = std::string(m) == "graph" ? 1 : 0;
    {
        // Domain slabs and growth tables come from the device's stream-ordered pool: admission and
        // retirement then queue behind running cycles instead of synchronising the device, and
        // freed slabs are reused by later admissions (the pool keeps what it has reserved until
        // this process ends).
        cudaMemPool_t mp;
        CUDA_OK(cudaDeviceGetDefaultMemPool(&mp, device));
        unsigned long long keep = ~0ull;
        CUDA_OK(cudaMemPoolSetAttribute(mp, cudaMemPoolAttrReleaseThreshold, &keep));
    }
    CUDA_OK(cudaMalloc(&dstate_, sizeof(PoolState)));
    CUDA_OK(cudaMalloc(&ddesc_, sizeof(DomainDesc) * (max_domains_ + 1)));
    CUDA_OK(cudaMemset(ddesc_, 0, sizeof(DomainDesc) * (max_domains_ + 1)));
    {
        // descriptor max_domains_ is a placeholder that is always finished
        DomainDesc ph;
        std::memset(&ph, 0, sizeof(ph));
        ph.done = 1;
        CUDA_OK(cudaMemcpy(ddesc_ + max_domains_, &ph, sizeof(ph), cudaMemcpyHostToDevice));
    }
    PoolState ps;
    std::memset(&ps, 0, sizeof(ps));
    for (int q = 0; q < 2; q++) {
        CUDA_OK(cudaMalloc(&ps.rec[q], capacity_ * sizeof(ActiveRec)));
        CUDA_OK(cudaMalloc(&ps.rdom[q], capacity_ * sizeof(unsigned int)));
        CUDA_OK(cudaMalloc(&ps.rstat[q], capacity_ * sizeof(unsigned int)));
        CUDA_OK(cudaMalloc(&ps.rmin2[q], capacity_ * sizeof(unsigned long long)));
    }
    // a shard takes the entries of 1/kShards of the warps: room for its share of the list plus slack
    ps.shard_cap = capacity_ / kShards + 8192;
    const size_t qn = (size_t)kShards * ps.shard_cap;
    CUDA_OK(cudaMalloc(&ps.tgt, qn * sizeof(unsigned long long)));
    CUDA_OK(cudaMalloc(&ps.qpos, qn * sizeof(unsigned int)));
    CUDA_OK(cudaMalloc(&ps.qcell, qn * sizeof(unsigned int)));
    CUDA_OK(cudaMalloc(&ps.qdom, qn * sizeof(unsigned int)));
    CUDA_OK(cudaMalloc(&ps.qmask, qn * sizeof(unsigned int)));
    CUDA_OK(cudaMalloc(&ps.qdl, qn * sizeof(float)));
    ps.capacity = capacity_;
    ps.cur = 0;
    ps.pending = 0;
    ps.n_domains = 0;
    ps.desc = ddesc_;
    CUDA_OK(cudaMemcpy(dstate_, &ps, sizeof(ps), cudaMemcpyHostToDevice));
    CUDA_OK(cudaMalloc(&census_buf_, sizeof(Census)));
}

Pool::~Pool() {
    cudaSetDevice(device_);
    cudaStreamSynchronize(S(stream_));
    if (graph_exec_)
        cudaGraphExecDestroy((cudaGraphExec_t)graph_exec_);
    for (auto &s : slots_) {
        for (void *p : s.allocs)
            cudaFree(p);
        if (s.growth)
            cudaFree(s.growth);
    }
    for (auto &kv : tables_) {
        cudaFree(kv.second.guv);
        cudaFree(kv.second.cdl_table);
    }
    if (dstate_) {
        PoolState ps;
        if (cudaMemcpy(&ps, dstate_, sizeof(ps), cudaMemcpyDeviceToHost) == cudaSuccess) {
            for (int q = 0; q < 2; q++) {
                cudaFree(ps.rec[q]);
                cudaFree(ps.rdom[q]);
                cudaFree(ps.rstat[q]);
                cudaFree(ps.rmin2[q]);
            }
            cudaFree(ps.tgt);
            cudaFree(ps.qpos);
            cudaFree(ps.qcell);
            cudaFree(ps.qdom);
            cudaFree(ps.qmask);
            cudaFree(ps.qdl);
        }
        cudaFree(dstate_);
    }
    cudaFree(ddesc_);
    cudaFree(census_buf_);
    if (copy_stream_)
        cudaStreamSynchronize(S(copy_stream_));
    for (int b = 0; b < 2; b++) {
        if (stage_[b])
            cudaFreeHost(stage_[b]);
        if (stage_ev_[b])
            cudaEventDestroy((cudaEvent_t)stage_ev_[b]);
    }
    cudaStreamDestroy(S(stream_));
    if (copy_stream_)
        cudaStreamDestroy(S(copy_stream_));
}

const DeviceTables &Pool::tables_for(const Problem &p) {
    auto it = tables_.find(p.cfg.orientation_file);
    if (it != tables_.end())
        return it->second;
    DeviceTables t;
    CUDA_OK(cudaMalloc(&t.guv, p.guv.size() * sizeof(float)));
    CUDA_OK(cudaMalloc(&t.cdl_table, p.cdl_table.size() * sizeof(float)));
    CUDA_OK(cudaMemcpy(t.guv, p.guv.data(), p.guv.size() * sizeof(float), cudaMemcpyHostToDevice));
    CUDA_OK(cudaMemcpy(t.cdl_table, p.cdl_table.data(), p.cdl_table.size() * sizeof(float), cudaMemcpyHostToDevice));
    h2d_bytes_ += (p.guv.size() + p.cdl_table.size()) * sizeof(float);
    return tables_[p.cfg.orientation_file] = t;
}

void Pool::push_desc(int slot) {
    // pageable source: staged before the call returns
    CUDA_OK(cudaMemcpyAsync(ddesc_ + slot, &host_desc_[slot], sizeof(DomainDesc), cudaMemcpyHostToDevice, S(stream_)));
}

void Pool::ensure_growth(int slot, long long needed) {
    SlotHost &s = slots_[slot];
    if (needed < s.growth_len)
        return;
    long long len = std::max<long long>(needed + 1, std::max<long long>(2LL * s.growth_len, 4096));
    if (len > INT_MAX / 2)
        throw Unsupported("growth table too long");
    // one table per distinct UndercoolingChange value, table c at c * len
    const Problem &p = *s.problem;
    const size_t n_tables = std::max<size_t>(1, p.du_values.size());
    std::vector<double> g(n_tables * (size_t)len);
    if (p.du_values.size() > 1) {
        for (size_t c = 0; c < n_tables; c++)
            build_growth_table(p, p.du_values[c], (int)len, g.data() + c * (size_t)len);
    }
    else {
        build_growth_table(p, p.du_value, (int)len, g.data());
    }
    double *d = nullptr;
    CUDA_OK(cudaMallocAsync((void **)&d, g.size() * sizeof(double), S(stream_)));
    CUDA_OK(cudaMemcpyAsync(d, g.data(), g.size() * sizeof(double), cudaMemcpyHostToDevice, S(stream_)));
    h2d_bytes_ += g.size() * sizeof(double);
    if (s.growth) {
        // queued work may still read the old table: it is freed in stream order after that work
        CUDA_OK(cudaFreeAsync(s.growth, S(stream_)));
    }
    s.growth = d;
    s.growth_len = (int)len;
    // patch only the table fields of the device descriptor
    DomainDesc &h = host_desc_[slot];
    h.growth = d;
    h.growth_len = (int)len;
    CUDA_OK(cudaMemcpyAsync((char *)(ddesc_ + slot) + offsetof(DomainDesc, growth), &h.growth, sizeof(h.growth),
                            cudaMemcpyHostToDevice, S(stream_)));
    CUDA_OK(cudaMemcpyAsync((char *)(ddesc_ + slot) + offsetof(DomainDesc, growth_len), &h.growth_len,
                            sizeof(h.growth_len), cudaMemcpyHostToDevice, S(stream_)));
}

// Named range on the host timeline for profilers (NVTX; inert when no tool is attached).
struct TraceRange {
    explicit TraceRange(const char *name) { nvtxRangePushA(name); }
    ~TraceRange() { nvtxRangePop(); }
    TraceRange(const TraceRange &) = delete;
    TraceRange &operator=(const TraceRange &) = delete;
};

int Pool::admit(std::shared_ptr<const Problem> pp, int check_mode) {
    TraceRange trace("exaca admit");
    CUDA_OK(cudaSetDevice(device_));
    const Problem &p = *pp;
    if (p.g.zbound_low != 0)
        throw Unsupported("active window must start at z = 0");
    size_t need = slot_bytes(p);
    if (bytes_in_use_ + need > budget_)
        throw AdmissionRefused("admission refused: HBM budget exceeded");
    int slot = -1;
    for (int s = 0; s < (int)slots_.size(); s++)
        if (!slots_[s].used) {
            slot = s;
            break;
        }
    if (slot < 0) {
        if ((int)slots_.size() >= max_domains_)
            throw AdmissionRefused("admission refused: too many domains");
        slot = (int)slots_.size();
        slots_.emplace_back();
        host_desc_.emplace_back();
    }
    SlotHost &s = slots_[slot];
    s = SlotHost();
    s.used = true;
    s.problem = pp;
    const Geometry &g = p.g;
    const int n_layers = p.cfg.number_of_layers;
    const bool multilayer = n_layers > 1;
    const bool classes = p.du_values.size() > 1;
    if (check_mode && p.cfg.simulation_type != "C")
        throw Unsupported("device-side termination covers type-C problems (types S and R jump cycles, stop at "
                          "finish time steps or change layers between launches): admit with device_check 0 "
                          "and run the plain path");
    const size_t N = g.domain_size, A = octahedron_cells(p), P = p.nuclei_loc.size();
    // every field of the slot in one allocation (256-byte aligned sub-arrays)
    size_t off = 0;
    auto carve = [&](size_t bytes) {
        size_t o = off;
        off += (std::max<size_t>(bytes, 16) + 255) & ~(size_t)255;
        return o;
    };
    const size_t o_ct = carve(N), o_gid = carve(N * 4), o_cts = carve(N * 4), o_ly = carve(N), o_du = carve(N * 4),
                 o_dl = carve(A * 4), o_doc = carve(A * 12), o_cdl = carve(A * 104), o_claim = carve(A * 8),
                 o_pos = carve(A * 4), o_nl = carve(P * 4), o_nt = carve(P * 4),
                 o_run = multilayer ? carve(N * 4) : 0, o_base = multilayer ? carve(N * 4) : 0,
                 o_cls = classes ? carve(N * 2) : 0;
    char *slab = nullptr;
    CUDA_OK(cudaMallocAsync((void **)&slab, off, S(stream_)));
    s.allocs.push_back(slab);
    s.bytes = off;
    DomainDesc d;
    std::memset(&d, 0, sizeof(d));
    d.ctype = (int8_t *)(slab + o_ct);
    d.gid = (int32_t *)(slab + o_gid);
    d.cts = (int32_t *)(slab + o_cts);
    d.layer = (int8_t *)(slab + o_ly);
    d.du = (float *)(slab + o_du);
    d.dl = (float *)(slab + o_dl);
    d.doc = (float *)(slab + o_doc);
    d.cdl = (float *)(slab + o_cdl);
    d.claim = (unsigned long long *)(slab + o_claim);
    d.pos = (unsigned int *)(slab + o_pos);
    d.cts_run = multilayer ? (int32_t *)(slab + o_run) : d.cts;
    d.nu_base = multilayer ? (int32_t *)(slab + o_base) : nullptr;
    d.du_class = classes ? (const uint16_t *)(slab + o_cls) : nullptr;
    int32_t *dnl = (int32_t *)(slab + o_nl);
    int32_t *dnt = (int32_t *)(slab + o_nt);
    // nuclei in time order; ties keep the reference's order (order does not change results)
    std::vector<int> order(P);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return p.nuclei_time[a] < p.nuclei_time[b]; });
    std::vector<int32_t> nl(P), nt(P);
    for (size_t q = 0; q < P; q++) {
        nl[q] = p.nuclei_loc[order[q]];
        nt[q] = p.nuclei_time[order[q]];
    }
    // host->device copies on the pool stream; pageable sources are staged before each call returns
    cudaStream_t st = S(stream_);
    if (p.dir.used) {
        // type C: the cell fields are made here from the plane CritTimeSteps, the substrate seeds and
        // the nuclei (a few KB cross PCIe instead of 14 bytes per cell)
        const size_t nk = p.dir.plane_cts.size(), na = p.dir.active.size(), nn = p.nuclei_loc.size();
        const size_t bytes = nk * 4 + na * 8 + nn * 4;
        // one upload: the 8-byte seed indices first (the allocation is 256-byte aligned), then the
        // 4-byte plane CritTimeSteps and nucleus indices
        std::vector<char> host(bytes);
        std::memcpy(host.data(), p.dir.active.data(), na * 8);
        std::memcpy(host.data() + na * 8, p.dir.plane_cts.data(), nk * 4);
        std::memcpy(host.data() + na * 8 + nk * 4, p.nuclei_loc.data(), nn * 4);
        char *dseed = nullptr;
        CUDA_OK(cudaMallocAsync((void **)&dseed, std::max<size_t>(bytes, 16), st));
        CUDA_OK(cudaMemcpyAsync(dseed, host.data(), bytes, cudaMemcpyHostToDevice, st));
        h2d_bytes_ += bytes;
        const long long *active = (const long long *)dseed;
        const int32_t *plane_cts = (const int32_t *)(dseed + na * 8);
        const int32_t *nuc = (const int32_t *)(dseed + na * 8 + nk * 4);
        const unsigned blocks = (unsigned)std::min<long long>((N + 255) / 256, (long long)num_sms_ * 16);
        k_fill_directional<<<blocks, 256, 0, st>>>(d.ctype, d.gid, d.cts, d.layer, d.du, (long long)N, g.mx, g.my,
                                                   g.nz, plane_cts, p.du_value);
        CUDA_OK(cudaGetLastError());
        const long long nseed = (long long)(na + nn);
        if (nseed)
            k_scatter_seeds<<<(unsigned)((nseed + 255) / 256), 256, 0, st>>>(d.ctype, d.gid, active, (long long)na,
                                                                             nuc, (long long)nn);
        CUDA_OK(cudaGetLastError());
        CUDA_OK(cudaFreeAsync(dseed, st));
    }
    else {
        CUDA_OK(cudaMemcpyAsync(d.ctype, p.cell_type.data(), N, cudaMemcpyHostToDevice, st));
        CUDA_OK(cudaMemcpyAsync(d.gid, p.grain_id.data(), N * 4, cudaMemcpyHostToDevice, st));
        CUDA_OK(cudaMemcpyAsync(d.cts, p.cts.data(), N * 4, cudaMemcpyHostToDevice, st));
        CUDA_OK(cudaMemcpyAsync(d.layer, p.layer_id.data(), N, cudaMemcpyHostToDevice, st));
        CUDA_OK(cudaMemcpyAsync(d.du, p.du.data(), N * 4, cudaMemcpyHostToDevice, st));
        h2d_bytes_ += N * 14;
    }
    CUDA_OK(cudaMemsetAsync(d.dl, 0, A * 4, st));
    CUDA_OK(cudaMemsetAsync(d.claim, 0xff, A * 8, st));
    CUDA_OK(cudaMemsetAsync(d.pos, 0xff, A * 4, st)); // kNoRecord
    if (multilayer)
        CUDA_OK(cudaMemsetAsync(d.nu_base, 0, N * 4, st));
    if (classes)
        CUDA_OK(cudaMemcpyAsync((void *)d.du_class, p.du_class.data(), N * 2, cudaMemcpyHostToDevice, st));
    if (P) {
        CUDA_OK(cudaMemcpyAsync(dnl, nl.data(), P * 4, cudaMemcpyHostToDevice, st));
        CUDA_OK(cudaMemcpyAsync(dnt, nt.data(), P * 4, cudaMemcpyHostToDevice, st));
    }
    h2d_bytes_ += (classes ? N * 2 : 0) + P * 8;
    const DeviceTables &tb = tables_for(p);
    d.guv = tb.guv;
    d.cdl_table = tb.cdl_table;
    d.nuc_loc = dnl;
    d.nuc_time = dnt;
    d.n_nuclei = (int)P;
    d.mx = g.mx;
    d.my = g.my;
    d.nz = g.nz;
    d.nz_active = g.nz_active;
    d.xoff = g.xoff;
    d.yoff = g.yoff;
    d.zbound_high = g.zbound_high;
    d.layer_no = 0;
    d.n_layers = n_layers;
    d.z_lo = g.zbound_low;
    d.z_end = g.zbound_low + g.nz_active;
    d.check_mode = check_mode;
    d.domain_size = g.domain_size;
    d.active_size = (long long)A;
    d.du_value = p.du_value;
    long long liquid = 0;
    int zero_du = 0, cts_max = INT_MIN;
    if (p.dir.used) {
        // every cell inside the wall ring is liquid except the substrate seeds
        liquid = (long long)(g.mx - 2) * (g.my - 2) * (g.nz - 2) - (long long)p.dir.active.size();
        zero_du = p.du_value == 0.0f ? 1 : 0;
        for (int32_t c : p.dir.plane_cts)
            cts_max = std::max(cts_max, c);
    }
    else {
        for (long i = 0; i < g.domain_size; i++) {
            int8_t t = p.cell_type[i];
            if (t == kLiquid && p.layer_id[i] == 0)
                liquid++;
            if ((t == kLiquid || t == kActive) && p.du[i] == 0.0f)
                zero_du = 1;
            cts_max = std::max(cts_max, p.cts[i]);
        }
    }
    d.liquid = liquid;
    d.zero_du = zero_du;
    d.cts_max = cts_max == INT_MIN ? INT_MAX : cts_max;
    host_desc_[slot] = d;
    push_desc(slot);
    if (multilayer) {
        k_layer_gate<<<num_sms_ * 4, 256, 0, st>>>(ddesc_ + slot);
        CUDA_OK(cudaGetLastError());
    }
    if (multilayer || classes) {
        static const int one = 1;
        CUDA_OK(cudaMemcpyAsync((char *)dstate_ + offsetof(PoolState, extras), &one, sizeof(int),
                                cudaMemcpyHostToDevice, st));
    }
    ensure_growth(slot, 4096);
    if (!p.voronoi_seeds.empty() || p.cfg.simulation_type != "C") {
        int nseeds = (int)(p.voronoi_seeds.size() / 3);
        int32_t *dseeds = nullptr;
        if (nseeds) {
            CUDA_OK(cudaMallocAsync((void **)&dseeds, p.voronoi_seeds.size() * 4, st));
            CUDA_OK(cudaMemcpyAsync(dseeds, p.voronoi_seeds.data(), p.voronoi_seeds.size() * 4,
                                    cudaMemcpyHostToDevice, st));
        }
        long long blocks = (g.domain_size + 255) / 256;
        k_voronoi<<<(unsigned)blocks, 256, 3 * 1024 * sizeof(int), st>>>(ddesc_ + slot, dseeds, nseeds,
                                                                         (float)(g.active_size));
        CUDA_OK(cudaGetLastError());
        if (dseeds)
            CUDA_OK(cudaFreeAsync(dseeds, st));
    }
    // register the domain, then build its initial active list in the list the next cycle consumes
    n_domains_ = std::max(n_domains_, slot + 1);
    CUDA_OK(cudaMemcpyAsync((char *)dstate_ + offsetof(PoolState, n_domains), &n_domains_, sizeof(int),
                            cudaMemcpyHostToDevice, st));
    k_init_active<<<num_sms_ * 4, 256, 0, st>>>(dstate_, slot, -1);
    CUDA_OK(cudaGetLastError());
    bytes_in_use_ += s.bytes;
    last_records_ = 0; // the list length is unknown until the next state read
    return slot;
}

void Pool::retire(int slot) {
    TraceRange trace("exaca retire");
    CUDA_OK(cudaSetDevice(device_));
    SlotHost &s = slots_.at(slot);
    if (!s.used)
        return;
    cudaStream_t st = S(stream_);
    // mark done and drop its list entries before the memory goes away
    int one = 1;
    CUDA_OK(cudaMemcpyAsync((char *)(ddesc_ + slot) + offsetof(DomainDesc, done), &one, sizeof(int),
                            cudaMemcpyHostToDevice, st));
    k_drop_domain<<<num_sms_ * 2, 256, 0, st>>>(dstate_, (unsigned)slot, (unsigned)max_domains_);
    CUDA_OK(cudaGetLastError());
    DomainDesc zero;
    std::memset(&zero, 0, sizeof(zero));
    zero.done = 1;
    host_desc_[slot] = zero;
    // the copies from host memory are staged before each call returns; everything below runs in
    // stream order after the cycles already queued, so nothing waits here
    CUDA_OK(cudaMemcpyAsync(ddesc_ + slot, &zero, sizeof(zero), cudaMemcpyHostToDevice, st));
    for (void *p : s.allocs)
        CUDA_OK(cudaFreeAsync(p, st));
    if (s.growth)
        CUDA_OK(cudaFreeAsync(s.growth, st));
    bytes_in_use_ -= s.bytes;
    s = SlotHost();
}

// One cooperative launch of k_cycles over n cycles (the grid is exactly the co-resident blocks).
void Pool::launch_persistent(int n) {
    cudaStream_t st = S(stream_);
    // the meeting point starts at zero arrivals (a launch that gave up waiting may have left some)
    CUDA_OK(cudaMemsetAsync((char *)dstate_ + offsetof(PoolState, bar_count), 0, 2 * sizeof(unsigned int), st));
    PoolState *ps = dstate_;
    // the domains still running at the last state read, when few (the one with most cells first);
    // one that ends during the launch is still started and returns at once, as in the spread start
    AliveSet alive{};
    for (int s = 0; s < (int)slots_.size() && alive.n >= 0; s++) {
        if (!slots_[s].used || host_desc_[s].done)
            continue;
        if (alive.n == kSerialDomains) {
            alive.n = -1;
            break;
        }
        alive.idx[alive.n++] = s;
    }
    for (int i = 1; i < alive.n; i++)
        if (host_desc_[alive.idx[i]].active_size > host_desc_[alive.idx[0]].active_size)
            std::swap(alive.idx[0], alive.idx[i]);
    void *args[] = {&ps, &n, &alive};
    // a sixteenth of the co-resident blocks for a list too short to fill them (fewer arrivals at
    // every grid-wide meeting; on a many-domain map measured faster below ~8e3 records, slower from
    // ~1.7e4, and the half grid slower than the full one from ~3e4 up)
    constexpr unsigned long long kSmallGridRecords = 1ull << 13;
    // run_plain before its trials: half of them below 2^17 records (its first launch, while the
    // list grows from the initial front)
    constexpr unsigned long long kHalfGridRecords = 1ull << 17;
    if (grid_fixed_)
        grid_div_ = grid_fixed_;
    else if (!grid_tuned_ && plain_run_)
        grid_div_ = (last_records_ > 0 && last_records_ < kHalfGridRecords) ? 2 : 1;
    else if (!grid_tuned_)
        grid_div_ = (last_records_ > 0 && last_records_ < kSmallGridRecords) ? 16 : 1;
    const int grid = std::max(1, grid_cycles_[variant_] / grid_div_);
    CUDA_OK(cudaLaunchCooperativeKernel(kStepKernel[variant_].cycles, dim3(grid), dim3(kBlock), args, 0, st));
    launches_ += 1;
}

// n cycles as separate pass kernels: the start of cycles 2..n runs in the last block of the
// previous capture pass, so a cycle costs three launches.
void Pool::launch_passes(int n) {
    if (n <= 0)
        return;
    cudaStream_t st = S(stream_);
    const StepKernels &K = kStepKernel[variant_];
    k_step_begin<<<1, kBlock, 0, st>>>(dstate_);
    for (int q = 0; q < n; q++) {
        K.grow<<<grid_grow_[variant_], kBlock, 0, st>>>(dstate_);
        k_claim<<<grid_claim_, kBlock, 0, st>>>(dstate_);
        if (q + 1 < n)
            K.capture_begin<<<grid_capture_[variant_], kBlock, 0, st>>>(dstate_);
        else
            K.capture_end<<<grid_capture_[variant_], kBlock, 0, st>>>(dstate_);
    }
    launches_ += 1 + 3ull * n;
}

void Pool::build_graph() {
    if (graph_exec_)
        return;
    graph_steps_ = 50;
    cudaStream_t st = S(stream_);
    cudaGraph_t graph;
    CUDA_OK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    const unsigned long long before = launches_;
    launch_passes(graph_steps_);
    launches_ = before;
    CUDA_OK(cudaStreamEndCapture(st, &graph));
    cudaGraphExec_t ex;
    CUDA_OK(cudaGraphInstantiate(&ex, graph, 0));
    CUDA_OK(cudaGraphDestroy(graph));
    graph_exec_ = ex;
}

void Pool::step(int n) {
    TraceRange trace("exaca step");
    if (n <= 0)
        return;
    cycles_launched_ += (unsigned long long)n;
    CUDA_OK(cudaSetDevice(device_));
    for (int s = 0; s < (int)slots_.size(); s++) {
        // a domain known to have ended executes no further cycle
        if (!slots_[s].used || host_desc_[s].done)
            continue;
        slots_[s].steps_launched += n;
        ensure_growth(s, slots_[s].steps_launched + 1);
    }
    if (step_mode_ == 0) {
        launch_persistent(n);
    }
    else {
        build_graph();
        cudaStream_t st = S(stream_);
        const int full = n / graph_steps_, rest = n % graph_steps_;
        for (int q = 0; q < full; q++)
            CUDA_OK(cudaGraphLaunch((cudaGraphExec_t)graph_exec_, st));
        launches_ += (unsigned long long)full * (1 + 3ull * graph_steps_);
        launch_passes(rest);
    }
    CUDA_OK(cudaGetLastError());
}

void Pool::sync_state() {
    CUDA_OK(cudaSetDevice(device_));
    cudaStream_t st = S(stream_);
    if (!host_desc_.empty())
        CUDA_OK(cudaMemcpyAsync(host_desc_.data(), ddesc_, sizeof(DomainDesc) * host_desc_.size(),
                                cudaMemcpyDeviceToHost, st));
    // the list counters (cnt[2], capacity, tombs, cur): the length of the list the next cycle reads
    constexpr size_t kCnt = offsetof(PoolState, cnt), kEnd = offsetof(PoolState, cur) + sizeof(int);
    unsigned char lists[kEnd - kCnt];
    CUDA_OK(cudaMemcpyAsync(lists, (char *)dstate_ + kCnt, sizeof(lists), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    unsigned long long cnt[2];
    int cur;
    std::memcpy(cnt, lists, sizeof(cnt));
    std::memcpy(&cur, lists + (offsetof(PoolState, cur) - kCnt), sizeof(cur));
    last_records_ = cnt[cur & 1];
}

int Pool::check_bounded_wait() {
    CUDA_OK(cudaSetDevice(device_));
    cudaStream_t st = S(stream_);
    CUDA_OK(cudaMemsetAsync((char *)dstate_ + offsetof(PoolState, bar_count), 0, 2 * sizeof(unsigned int), st));
    PoolState *ps = dstate_;
    void *args[] = {&ps};
    CUDA_OK(cudaLaunchCooperativeKernel((const void *)k_meet_probe, dim3(2), dim3(kBlock), args, 0, st));
    launches_ += 1;
    const int flags = pool_error();
    // the pool carries on: no flag and a meeting point with no arrivals
    const int zero = 0;
    CUDA_OK(cudaMemcpyAsync((char *)dstate_ + offsetof(PoolState, error), &zero, sizeof(int), cudaMemcpyHostToDevice,
                            st));
    CUDA_OK(cudaMemsetAsync((char *)dstate_ + offsetof(PoolState, bar_count), 0, 2 * sizeof(unsigned int), st));
    CUDA_OK(cudaStreamSynchronize(st));
    return flags;
}

int Pool::pool_error() {
    int e = 0;
    CUDA_OK(cudaMemcpyAsync(&e, (char *)dstate_ + offsetof(PoolState, error), sizeof(int), cudaMemcpyDeviceToHost,
                            S(stream_)));
    CUDA_OK(cudaStreamSynchronize(S(stream_)));
    return e;
}

unsigned long long Pool::list_count() {
    PoolState ps;
    CUDA_OK(cudaMemcpyAsync(&ps, dstate_, sizeof(ps), cudaMemcpyDeviceToHost, S(stream_)));
    CUDA_OK(cudaStreamSynchronize(S(stream_)));
    return ps.cnt[ps.pending];
}

PoolStats Pool::stats() {
    PoolState ps;
    CUDA_OK(cudaMemcpyAsync(&ps, dstate_, sizeof(ps), cudaMemcpyDeviceToHost, S(stream_)));
    CUDA_OK(cudaStreamSynchronize(S(stream_)));
    PoolStats r;
    std::memset(&r, 0, sizeof(r));
    r.cycles = cycles_launched_;
    r.launches = launches_;
    r.h2d_bytes = h2d_bytes_;
    r.d2h_bytes = d2h_bytes_;
    for (int q = 0; q < kStatShards; q++) {
        r.listed += ps.stat[q][kStatListed];
        r.grown += ps.stat[q][kStatGrown];
        r.captured += ps.stat[q][kStatCaptured];
        r.nucleated += ps.stat[q][kStatNucleated];
        r.claims += ps.stat[q][kStatClaims];
        r.row_reads += ps.stat[q][kStatRowReads];
        r.dropped += ps.stat[q][kStatDropped];
        r.fresh += ps.stat[q][kStatFresh];
        r.rechecks += ps.stat[q][kStatRechecks];
        r.flagged += ps.stat[q][kStatFlagged];
    }
    return r;
}

KernelTimes Pool::profile_cycles(int n) {
    CUDA_OK(cudaSetDevice(device_));
    KernelTimes kt;
    if (n <= 0)
        return kt;
    for (int s = 0; s < (int)slots_.size(); s++) {
        if (!slots_[s].used)
            continue;
        slots_[s].steps_launched += n;
        ensure_growth(s, slots_[s].steps_launched + 1);
    }
    cudaStream_t st = S(stream_);
    cudaEvent_t ev[5];
    for (auto &e : ev)
        CUDA_OK(cudaEventCreate(&e));
    for (int q = 0; q < n; q++) {
        CUDA_OK(cudaEventRecord(ev[0], st));
        k_step_begin<<<1, kBlock, 0, st>>>(dstate_);
        CUDA_OK(cudaEventRecord(ev[1], st));
        kStepKernel[variant_].grow<<<grid_grow_[variant_], kBlock, 0, st>>>(dstate_);
        CUDA_OK(cudaEventRecord(ev[2], st));
        k_claim<<<grid_claim_, kBlock, 0, st>>>(dstate_);
        CUDA_OK(cudaEventRecord(ev[3], st));
        kStepKernel[variant_].capture_end<<<grid_capture_[variant_], kBlock, 0, st>>>(dstate_);
        CUDA_OK(cudaEventRecord(ev[4], st));
        CUDA_OK(cudaEventSynchronize(ev[4]));
        float t[4];
        for (int k = 0; k < 4; k++)
            CUDA_OK(cudaEventElapsedTime(&t[k], ev[k], ev[k + 1]));
        kt.begin_ms += t[0];
        kt.grow_ms += t[1];
        kt.claim_ms += t[2];
        kt.capture_ms += t[3];
    }
    CUDA_OK(cudaGetLastError());
    for (auto &e : ev)
        CUDA_OK(cudaEventDestroy(e));
    kt.cycles = n;
    cycles_launched_ += (unsigned long long)n;
    launches_ += 4ull * n;
    return kt;
}

void Pool::profile_persistent(int n, double us[7]) {
    for (int k = 0; k < 7; k++)
        us[k] = 0;
    if (n <= 0)
        return;
    CUDA_OK(cudaSetDevice(device_));
    cudaStream_t st = S(stream_);
    const size_t words = 3 * (3 * (size_t)n + 1);
    unsigned long long *dtl = nullptr;
    CUDA_OK(cudaMalloc(&dtl, words * sizeof(unsigned long long)));
    CUDA_OK(cudaMemsetAsync(dtl, 0, words * sizeof(unsigned long long), st));
    CUDA_OK(cudaMemcpyAsync((char *)dstate_ + offsetof(PoolState, timeline), &dtl, sizeof(dtl),
                            cudaMemcpyHostToDevice, st));
    step(n);
    unsigned long long *none = nullptr;
    CUDA_OK(cudaMemcpyAsync((char *)dstate_ + offsetof(PoolState, timeline), &none, sizeof(none),
                            cudaMemcpyHostToDevice, st));
    std::vector<unsigned long long> tl(words);
    CUDA_OK(cudaMemcpyAsync(tl.data(), dtl, words * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    CUDA_OK(cudaFree(dtl));
    // meeting points 3c+1, 3c+2, 3c+3 close cycle c's growth (with the blocks' own claims), global
    // claim and capture passes; 3c+2 is skipped (all zero) in cycles without a queue overflow
    for (int c = 0; c < n; c++) {
        const unsigned long long *prev = &tl[3 * (3 * c)], *m1 = &tl[3 * (3 * c + 1)], *m2 = &tl[3 * (3 * c + 2)],
                                 *m3 = &tl[3 * (3 * c + 3)];
        us[0] += (double)(m1[0] - prev[2]);
        us[1] += (double)(m1[1] - prev[2]);
        const unsigned long long *before_capture = m1;
        if (m2[2]) {
            us[2] += (double)(m2[0] - m1[2]);
            us[3] += (double)(m2[1] - m1[2]);
            before_capture = m2;
        }
        us[4] += (double)(m3[0] - before_capture[2]);
        us[5] += (double)(m3[1] - before_capture[2]);
        us[6] += (double)(m3[2] - m3[1]);
    }
    for (int k = 0; k < 7; k++)
        us[k] /= 1e3 * n;
}

void Pool::set_config(int config) {
    apply_config(config);
    config_fixed_ = true;
}

void Pool::set_grid(int divisor) {
    if (divisor < 0 || divisor > 32)
        throw std::invalid_argument("grid divisor must be 0 (automatic) or 1-32");
    grid_fixed_ = divisor;
}

int Pool::plain_tune(int n) {
    int best = variant_, best_div = 1;
    double best_ms = 1e300;
    grid_tuned_ = true;
    // the half grid only for lists that are not clearly long (it measured 25 % slower at ~1e6
    // records, where its trials would cost more than they can find)
    const int min_div = grid_fixed_ ? grid_fixed_ : 1;
    const int max_div = grid_fixed_ ? grid_fixed_ : (last_records_ < (1ull << 19) ? 2 : 1);
    for (int div = min_div; div <= max_div; div++)
        for (int v = 0; v < kStepVariants; v++) {
            apply_config(v);
            grid_div_ = div;
            const double ms = timed_step(n);
            if (ms < best_ms) {
                best_ms = ms;
                best = v;
                best_div = div;
            }
        }
    apply_config(best);
    grid_div_ = best_div;
    return (max_div - min_div + 1) * kStepVariants * n;
}

void Pool::apply_config(int config) {
    if (config < 0 || config >= kStepConfigs)
        throw std::invalid_argument("step configuration out of range");
    const int mode = config / kStepVariants, variant = config % kStepVariants;
    if (variant != variant_ && graph_exec_) {
        CUDA_OK(cudaStreamSynchronize(S(stream_)));
        CUDA_OK(cudaGraphExecDestroy((cudaGraphExec_t)graph_exec_));
        graph_exec_ = nullptr;
    }
    step_mode_ = mode;
    variant_ = variant;
}

int Pool::autotune(int trial_cycles, double *ms_per_cycle) {
    int best = config();
    double best_ms = 1e300;
    for (int c = 0; c < kStepConfigs; c++) {
        apply_config(c);
        if (step_mode_ == 1)
            build_graph(); // outside the timed trial
        const double ms = timed_step(trial_cycles) / std::max(trial_cycles, 1);
        if (ms_per_cycle)
            ms_per_cycle[c] = ms;
        if (ms < best_ms) {
            best_ms = ms;
            best = c;
        }
    }
    set_config(best);
    return best;
}

long long Pool::run_all(int chunk, long long max_cycles) {
    TraceRange trace("exaca run_all");
    if (chunk <= 0)
        throw std::invalid_argument("chunk must be positive");
    long long stepped = 0;
    while (true) {
        sync_state();
        bool all_done = true;
        for (int s = 0; s < (int)slots_.size(); s++) {
            if (!slots_[s].used)
                continue;
            const DomainDesc &d = host_desc_[s];
            if (d.error)
                throw DeviceError("device error flags " + std::to_string(d.error) + " in slot " + std::to_string(s));
            if (!d.check_mode)
                throw std::invalid_argument("slot " + std::to_string(s) + " was admitted without device termination");
            all_done = all_done && d.done;
        }
        const int perr = pool_error();
        if (perr)
            throw DeviceError("pool error flags " + std::to_string(perr));
        if (all_done)
            return stepped;
        if (stepped >= max_cycles)
            throw DeviceError("domains still running after " + std::to_string(stepped) + " cycles");
        step(chunk);
        stepped += chunk;
    }
}

double Pool::timed_step(int n) {
    CUDA_OK(cudaSetDevice(device_));
    cudaStream_t st = S(stream_);
    cudaEvent_t ev[2];
    for (auto &e : ev)
        CUDA_OK(cudaEventCreate(&e));
    CUDA_OK(cudaEventRecord(ev[0], st));
    step(n);
    CUDA_OK(cudaEventRecord(ev[1], st));
    CUDA_OK(cudaEventSynchronize(ev[1]));
    float ms = 0;
    CUDA_OK(cudaEventElapsedTime(&ms, ev[0], ev[1]));
    for (auto &e : ev)
        CUDA_OK(cudaEventDestroy(e));
    return ms;
}

long long Pool::liquid(int slot) const {
    const DomainDesc &d = host_desc_.at(slot);
    long long v = d.liquid;
    for (int q = 0; q < kLiquidShards; q++)
        v += d.liquid_shard[q];
    return v;
}

Census Pool::census(int slot) {
    CUDA_OK(cudaSetDevice(device_));
    cudaStream_t st = S(stream_);
    Census init;
    std::memset(&init, 0, sizeof(init));
    init.next_cts = ULLONG_MAX;
    CUDA_OK(cudaMemcpyAsync(census_buf_, &init, sizeof(init), cudaMemcpyHostToDevice, st));
    k_census<<<num_sms_ * 4, 256, 0, st>>>(ddesc_ + slot, (Census *)census_buf_);
    CUDA_OK(cudaGetLastError());
    Census out;
    CUDA_OK(cudaMemcpyAsync(&out, census_buf_, sizeof(out), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    return out;
}

void Pool::set_cycle(int slot, int cycle) {
    sync_state();
    DomainDesc &h = host_desc_[slot];
    if (cycle > h.cycle) {
        if (h.n_jumps >= kMaxJumps)
            throw Unsupported("too many cycle jumps");
        h.jump_lo[h.n_jumps] = h.cycle;
        h.jump_hi[h.n_jumps] = cycle;
        h.n_jumps++;
    }
    h.cycle = cycle;
    // only this slot's dynamic fields change; nothing else is in flight on the stream
    push_desc(slot);
}

void Pool::next_layer(int slot, std::string &log) {
    TraceRange trace("exaca next_layer");
    // src/runCA.cpp:344-405: DomainShiftAndResize, then LayerSetup on the moved window
    CUDA_OK(cudaSetDevice(device_));
    cudaStream_t st = S(stream_);
    sync_state();
    DomainDesc d = host_desc_.at(slot);
    if (d.layer_no + 1 >= d.n_layers || !d.nu_base)
        throw std::logic_error("next_layer: the slot has no further layer");
    const unsigned blocks = (unsigned)num_sms_ * 4;
    k_layer_base<<<blocks, 256, 0, st>>>(ddesc_ + slot);
    CUDA_OK(cudaGetLastError());
    int bounds[2] = {INT_MAX, INT_MIN};
    int *dbounds = nullptr;
    CUDA_OK(cudaMalloc(&dbounds, sizeof(bounds)));
    CUDA_OK(cudaMemcpyAsync(dbounds, bounds, sizeof(bounds), cudaMemcpyHostToDevice, st));
    k_layer_bounds<<<blocks, 256, 0, st>>>(ddesc_ + slot, d.layer_no + 1, dbounds);
    CUDA_OK(cudaGetLastError());
    CUDA_OK(cudaMemcpyAsync(bounds, dbounds, sizeof(bounds), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    CUDA_OK(cudaFree(dbounds));
    // the new bottom is one plane below the lowest active cell, the new top the highest cell of the
    // next layer (src/CAinitialize.cpp:2776-2820)
    if (bounds[0] == INT_MAX || bounds[1] == INT_MIN || bounds[0] - 1 > bounds[1] || bounds[1] >= d.nz)
        throw DeviceError("layer change: no active cell or no cell of the next layer");
    const int z_lo = bounds[0] - 1, z_hi = bounds[1];
    std::ostringstream s;
    s << "New domain bottom at Z = " << z_lo << ", a shift of " << z_lo - d.z_lo << " cells\n";
    s << "New domain top at Z = " << z_hi << "\n";
    s << "New active domain height is " << z_hi - z_lo + 1 << "\n";
    s << "Resize executed\n";
    d.layer_no += 1;
    d.z_lo = z_lo;
    d.z_end = z_hi + 1;
    d.nz_active = z_hi - z_lo + 1;
    d.zbound_high = z_hi;
    d.cycle = 0;
    d.nuc_cursor = 0;
    d.nn = 0;
    d.n_jumps = 0;
    host_desc_[slot] = d;
    push_desc(slot);
    k_layer_gate<<<blocks, 256, 0, st>>>(ddesc_ + slot);
    CUDA_OK(cudaGetLastError());
    // LayerSetup: the records of the ended layer leave the list (re-labelled to the pool's finished
    // placeholder domain, dropped by the next growth pass); the window's octahedron arrays start from
    // zero (src/CAinitialize.cpp:2850-2852); every active cell of the new window gets a fresh
    // octahedron and a record
    k_drop_domain<<<num_sms_ * 2, 256, 0, st>>>(dstate_, (unsigned)slot, (unsigned)max_domains_);
    CUDA_OK(cudaGetLastError());
    CUDA_OK(cudaMemsetAsync(d.pos, 0xff, (size_t)d.active_size * 4, st));
    {
        const size_t plane = (size_t)d.mx * d.my, o = plane * d.z_lo, n = plane * (d.z_end - d.z_lo);
        CUDA_OK(cudaMemsetAsync(d.dl + o, 0, n * 4, st));
        CUDA_OK(cudaMemsetAsync(d.doc + 3 * o, 0, n * 12, st));
        CUDA_OK(cudaMemsetAsync(d.cdl + 26 * o, 0, n * 104, st));
    }
    k_init_active<<<num_sms_ * 4, 256, 0, st>>>(dstate_, slot, -1);
    CUDA_OK(cudaGetLastError());
    s << "New layer setup, GN dimensions are " << d.mx << " " << 0 << " " << d.nz_active << "\n";
    s << "New layer ghost nodes initialized\n";
    log += s.str();
}

void Pool::copy_out_raw(int slot, int32_t *grain_id, int8_t *cell_type) {
    CUDA_OK(cudaSetDevice(device_));
    const DomainDesc &d = host_desc_.at(slot);
    size_t N = slots_.at(slot).problem->g.domain_size;
    cudaStream_t st = S(stream_);
    to_host({{grain_id, d.gid, N * 4, false}, {cell_type, d.ctype, N, false}}, stream_);
    d2h_bytes_ += (grain_id ? N * 4 : 0) + (cell_type ? N : 0);
    CUDA_OK(cudaStreamSynchronize(st));
}

void Pool::flush_records() {
    CUDA_OK(cudaSetDevice(device_));
    k_flush_records<<<num_sms_ * 2, 256, 0, S(stream_)>>>(dstate_);
    CUDA_OK(cudaGetLastError());
    CUDA_OK(cudaStreamSynchronize(S(stream_)));
}

void Pool::copy_octahedra(int slot, float *dl, float *doc, float *cdl) {
    flush_records();
    const DomainDesc &d = host_desc_.at(slot);
    // the current layer's window (the whole allocation's prefix for single-layer problems)
    const size_t plane = (size_t)d.mx * d.my, o = plane * d.z_lo, A = plane * (d.z_end - d.z_lo);
    cudaStream_t st = S(stream_);
    to_host({{dl, d.dl + o, A * 4, false}, {doc, d.doc + 3 * o, A * 12, false}, {cdl, d.cdl + 26 * o, A * 104, false}},
            stream_);
    d2h_bytes_ += (dl ? A * 4 : 0) + (doc ? A * 12 : 0) + (cdl ? A * 104 : 0);
    CUDA_OK(cudaStreamSynchronize(st));
}

void Pool::copy_out(int slot, int32_t *grain_id, int32_t *cell_type) {
    TraceRange trace("exaca copy_out");
    if (!cell_type) {
        copy_out_raw(slot, grain_id, nullptr);
        return;
    }
    // CellType is widened to int32 on the device (in stream order after the cycles); both fields
    // then go to the caller's buffers as one DMA each when those are page-locked, else through the
    // pinned staging pieces
    CUDA_OK(cudaSetDevice(device_));
    const DomainDesc &d = host_desc_.at(slot);
    const size_t N = slots_.at(slot).problem->g.domain_size;
    cudaStream_t st = S(stream_);
    int32_t *wide = nullptr;
    CUDA_OK(cudaMallocAsync((void **)&wide, std::max<size_t>(N * 4, 16), st));
    const unsigned blocks = (unsigned)std::min<size_t>((N + 255) / 256, (size_t)num_sms_ * 16);
    k_widen_types<<<blocks, 256, 0, st>>>(d.ctype, wide, (long long)N);
    CUDA_OK(cudaGetLastError());
    to_host({{grain_id, d.gid, N * 4, false}, {cell_type, wide, N * 4, false}}, stream_);
    CUDA_OK(cudaFreeAsync(wide, st));
    CUDA_OK(cudaStreamSynchronize(st));
    d2h_bytes_ += (grain_id ? N * 4 : 0) + N * 4;
}

void Pool::copy_out_concurrent(int slot, int32_t *grain_id, int32_t *cell_type) {
    TraceRange trace("exaca copy_out_concurrent");
    CUDA_OK(cudaSetDevice(device_));
    const SlotHost &s = slots_.at(slot);
    const DomainDesc &d = host_desc_.at(slot);
    if (!s.used || !(d.done || s.finished))
        throw std::invalid_argument("copy_out_concurrent: the slot's domain has not ended");
    if (!copy_stream_) {
        cudaStream_t cs;
        CUDA_OK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        copy_stream_ = cs;
    }
    // The domain's GrainID and CellType are final (an ended domain's records only leave the list),
    // and the host saw that state, so the copies need no ordering against the pool stream. Copy
    // engines only: no kernel runs beside the persistent cooperative one.
    // CellType is widened on the host as it leaves the staging pieces.
    cudaStream_t cs = S(copy_stream_);
    const size_t N = s.problem->g.domain_size;
    to_host({{grain_id, d.gid, N * 4, false}, {cell_type, d.ctype, N, true}}, copy_stream_);
    CUDA_OK(cudaStreamSynchronize(cs));
    d2h_bytes_ += (grain_id ? N * 4 : 0) + (cell_type ? N : 0);
}

int Pool::run_plain(int slot, std::string &log, double *nucl_s, double *capture_s) {
    TraceRange trace("exaca run_plain");
    // its own grid rule until its trials choose, and the grid they choose holds for this run only
    // (the short-list rule of chunked stepping would hold a small domain's first 1000 cycles, while
    // its list grows from the initial front, on a sixteenth of the blocks)
    struct GridReset {
        bool &tuned, &plain;
        ~GridReset() { tuned = plain = false; }
    } grid_reset{grid_tuned_, plain_run_};
    plain_run_ = true;
    // src/runCA.cpp:282-411: the layer loop, each layer's cycles until no liquid of the layer is left
    const Problem &p = *slots_.at(slot).problem;
    const bool type_r = p.cfg.simulation_type == "R";
    const bool jump_type = p.cfg.simulation_type == "S" || type_r;
    auto t0 = std::chrono::steady_clock::now();
    auto t_layer = t0;
    cudaEvent_t ev0, ev1;
    CUDA_OK(cudaEventCreate(&ev0));
    CUDA_OK(cudaEventCreate(&ev1));
    CUDA_OK(cudaEventRecord(ev0, S(stream_)));
    sync_state();
    int cycle = host_desc_[slot].cycle;
    constexpr int kTuneCycles = 50;
    while (true) {
        int n = 1000 - (cycle % 1000);
        if (!config_fixed_ && cycle % 4000 == 1000 && n == 1000) {
            // the persistent configuration's speed depends on the domain's active front: time each
            // launch shape with the full and the half grid for kTuneCycles real cycles at cycle 1000
            // and every 4000 cycles after; the results do not depend on it
            n -= plain_tune(kTuneCycles);
        }
        step(n);
        sync_state();
        const DomainDesc &d = host_desc_[slot];
        int perr = pool_error();
        if (d.error || perr) {
            std::ostringstream e;
            e << "device error flags: domain " << d.error << " pool " << perr;
            throw DeviceError(e.str());
        }
        cycle = d.cycle;
        Census c = census(slot);
        std::ostringstream s;
        s << "cycle = " << cycle << " Superheated liquid cells = " << c.superheated
          << " Undercooled liquid cells = " << c.undercooled << " Number of nucleation events this layer " << d.nn
          << " Remaining liquid cells in future layers of this simulation = " << c.remaining << "\n";
        log += s.str();
        bool xswitch = c.superheated + c.undercooled == 0;
        if (!xswitch && jump_type && c.undercooled == 0) {
            unsigned long long next = c.next_cts;
            if ((next - (unsigned long long)(long long)cycle) > 5000) {
                int nc = (int)(next - 1);
                set_cycle(slot, nc);
                cycle = nc;
                log += "Jumping to cycle " + std::to_string(cycle + 1) + "\n";
            }
            // type R ends a layer at its finish time step (src/CAupdate.cpp:818-819)
            if (type_r && cycle >= p.finish_time_step.at(d.layer_no))
                xswitch = true;
        }
        if (xswitch) {
            if (d.layer_no + 1 >= d.n_layers)
                break;
            const int layer = d.layer_no;
            next_layer(slot, log);
            double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_layer).count();
            t_layer = std::chrono::steady_clock::now();
            std::ostringstream s2;
            s2 << "Time for layer number " << layer << " was " << secs << " s, starting layer " << layer + 1 << "\n";
            log += s2.str();
            cycle = 0;
            continue;
        }
    }
    CUDA_OK(cudaEventRecord(ev1, S(stream_)));
    CUDA_OK(cudaEventSynchronize(ev1));
    float ms = 0;
    CUDA_OK(cudaEventElapsedTime(&ms, ev0, ev1));
    last_run_ms_ = ms;
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (nucl_s)
        *nucl_s = 0.0;
    if (capture_s)
        *capture_s = secs;
    slots_[slot].finished = true;
    return cycle;
}

// ---------------------------------------------------------------------------------------------
// Grain statistics (analysis/src/GAprint.cpp:17-198) on the device: per region cell, melted count,
// misorientation of its grain's orientation to +Z (table built on the host with the reference's
// libm acos), its 1-degree histogram, nucleated cells, GrainID range; then distinct GrainIDs via a
// bitmap over that range.
struct GrainAcc {
    unsigned long long melted, nucleated, top_melted;
    double mis, mis_top;
    unsigned long long hist[kMisorientationBins];
    int gmin, gmax;
};

struct Region {
    int x0, x1, y0, y1, z0, z1, mx, my;
    __device__ __forceinline__ long long count() const {
        return (long long)(x1 - x0 + 1) * (y1 - y0 + 1) * (z1 - z0 + 1);
    }
    // q-th region cell: (k, i, j) of the .vtk grid -> rank-local index (ghost ring offset 1)
    __device__ __forceinline__ long long cell(long long q, int &k) const {
        const long long ny_r = y1 - y0 + 1, nx_r = x1 - x0 + 1;
        const long long j = q % ny_r, t = q / ny_r;
        const long long i = t % nx_r;
        k = (int)(t / nx_r) + z0;
        return (long long)k * mx * my + (i + x0 + 1) * my + (j + y0 + 1);
    }
};

__global__ void __launch_bounds__(kBlock) k_grain_region(const int32_t *gid, const int8_t *melted, const float *mis,
                                                         Region R, GrainAcc *acc) {
    __shared__ unsigned long long s_hist[kMisorientationBins];
    for (int b = threadIdx.x; b < kMisorientationBins; b += blockDim.x)
        s_hist[b] = 0;
    __syncthreads();
    unsigned long long m = 0, nuc = 0, top = 0;
    double ms = 0, mt = 0;
    int gmin = INT_MAX, gmax = INT_MIN;
    const long long n = R.count();
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        int k;
        const long long c = R.cell(q, k);
        const int g = gid[c];
        gmin = min(gmin, g);
        gmax = max(gmax, g);
        if (g < 0)
            nuc++;
        if (melted[c] == 1) {
            int ori = (abs(g) - 1) % 10000;
            if (ori < 0)
                ori += 10000;
            const float a = mis[ori];
            m++;
            ms += a;
            atomicAdd(&s_hist[min((int)a, kMisorientationBins - 1)], 1ull);
            if (k == R.z1) {
                top++;
                mt += a;
            }
        }
    }
    for (int o = 16; o; o >>= 1) {
        m += __shfl_down_sync(0xffffffffu, m, o);
        nuc += __shfl_down_sync(0xffffffffu, nuc, o);
        top += __shfl_down_sync(0xffffffffu, top, o);
        ms += __shfl_down_sync(0xffffffffu, ms, o);
        mt += __shfl_down_sync(0xffffffffu, mt, o);
        gmin = min(gmin, __shfl_down_sync(0xffffffffu, gmin, o));
        gmax = max(gmax, __shfl_down_sync(0xffffffffu, gmax, o));
    }
    if ((threadIdx.x & 31) == 0) {
        if (m)
            atomicAdd(&acc->melted, m);
        if (nuc)
            atomicAdd(&acc->nucleated, nuc);
        if (top)
            atomicAdd(&acc->top_melted, top);
        if (ms != 0)
            atomicAdd(&acc->mis, ms);
        if (mt != 0)
            atomicAdd(&acc->mis_top, mt);
        atomicMin(&acc->gmin, gmin);
        atomicMax(&acc->gmax, gmax);
    }
    __syncthreads();
    for (int b = threadIdx.x; b < kMisorientationBins; b += blockDim.x)
        if (s_hist[b])
            atomicAdd(&acc->hist[b], s_hist[b]);
}

__global__ void k_grain_bits(const int32_t *gid, Region R, int gmin, unsigned long long *bits) {
    const long long n = R.count();
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        int k;
        const long long off = (long long)gid[R.cell(q, k)] - gmin;
        atomicOr(bits + (off >> 6), 1ull << (off & 63));
    }
}

__global__ void k_popcount(const unsigned long long *bits, long long nwords, unsigned long long *count) {
    unsigned long long c = 0;
    for (long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x; w < nwords; w += (long long)gridDim.x * blockDim.x)
        c += __popcll(bits[w]);
    for (int o = 16; o; o >>= 1)
        c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c)
        atomicAdd(count, c);
}

GrainStats Pool::grain_stats(int slot, const int *region) {
    CUDA_OK(cudaSetDevice(device_));
    if (!slot_used(slot))
        throw std::invalid_argument("bad slot");
    const Problem &p = *slots_[slot].problem;
    materialize_fields(p);
    const Geometry &g = p.g;
    Region R;
    if (region) {
        R.x0 = region[0], R.x1 = region[1], R.y0 = region[2], R.y1 = region[3], R.z0 = region[4], R.z1 = region[5];
    }
    else {
        R.x0 = 1, R.x1 = g.nx - 2, R.y0 = 1, R.y1 = g.ny - 2, R.z0 = 1, R.z1 = g.nz - 2;
    }
    if (R.x0 < 0 || R.x1 >= g.nx || R.y0 < 0 || R.y1 >= g.ny || R.z0 < 0 || R.z1 >= g.nz || R.x0 > R.x1 ||
        R.y0 > R.y1 || R.z0 > R.z1)
        throw std::invalid_argument("region outside the domain");
    R.mx = g.mx;
    R.my = g.my;
    // per-orientation misorientation to +Z with the reference's expression (GAprint.cpp:38-46)
    std::vector<float> mis(kNumOrientations);
    for (int n = 0; n < kNumOrientations; n++) {
        double amin = 62.7;
        for (int ll = 0; ll < 3; ll++) {
            // double acos of the float component, as the reference's unqualified call on a float
            double a = std::abs((180 / M_PI) * std::acos((double)p.guv[9 * n + 3 * ll + 2]));
            if (a < amin)
                amin = a;
        }
        mis[n] = (float)amin;
    }
    cudaStream_t st = S(stream_);
    const size_t N = g.domain_size;
    int8_t *dmel = nullptr;
    float *dmis = nullptr;
    GrainAcc *dacc = nullptr;
    unsigned long long *bits = nullptr, *dcount = nullptr;
    GrainStats out;
    try {
        CUDA_OK(cudaMalloc(&dmel, N));
        CUDA_OK(cudaMalloc(&dmis, mis.size() * sizeof(float)));
        CUDA_OK(cudaMalloc(&dacc, sizeof(GrainAcc)));
        CUDA_OK(cudaMalloc(&dcount, sizeof(unsigned long long)));
        GrainAcc init;
        std::memset(&init, 0, sizeof(init));
        init.gmin = INT_MAX;
        init.gmax = INT_MIN;
        CUDA_OK(cudaMemcpyAsync(dmel, p.melted.data(), N, cudaMemcpyHostToDevice, st));
        CUDA_OK(cudaMemcpyAsync(dmis, mis.data(), mis.size() * sizeof(float), cudaMemcpyHostToDevice, st));
        CUDA_OK(cudaMemcpyAsync(dacc, &init, sizeof(init), cudaMemcpyHostToDevice, st));
        CUDA_OK(cudaMemsetAsync(dcount, 0, sizeof(unsigned long long), st));
        k_grain_region<<<num_sms_ * 4, kBlock, 0, st>>>(host_desc_[slot].gid, dmel, dmis, R, dacc);
        CUDA_OK(cudaGetLastError());
        GrainAcc acc;
        CUDA_OK(cudaMemcpyAsync(&acc, dacc, sizeof(acc), cudaMemcpyDeviceToHost, st));
        CUDA_OK(cudaStreamSynchronize(st));
        const long long range = (long long)acc.gmax - acc.gmin + 1;
        const long long nwords = (range + 63) / 64;
        CUDA_OK(cudaMalloc(&bits, nwords * 8));
        CUDA_OK(cudaMemsetAsync(bits, 0, nwords * 8, st));
        k_grain_bits<<<num_sms_ * 4, kBlock, 0, st>>>(host_desc_[slot].gid, R, acc.gmin, bits);
        k_popcount<<<num_sms_ * 2, kBlock, 0, st>>>(bits, nwords, dcount);
        CUDA_OK(cudaGetLastError());
        unsigned long long count = 0;
        CUDA_OK(cudaMemcpyAsync(&count, dcount, sizeof(count), cudaMemcpyDeviceToHost, st));
        CUDA_OK(cudaStreamSynchronize(st));
        out.region_cells = (long long)(R.x1 - R.x0 + 1) * (R.y1 - R.y0 + 1) * (R.z1 - R.z0 + 1);
        out.melted_cells = (long long)acc.melted;
        out.nucleated_cells = (long long)acc.nucleated;
        out.top_melted = (long long)acc.top_melted;
        out.n_grains = (long long)count;
        out.misorientation_sum = acc.mis;
        out.misorientation_top_sum = acc.mis_top;
        out.deltax = p.cfg.deltax;
        for (int b = 0; b < kMisorientationBins; b++)
            out.hist[b] = acc.hist[b];
    }
    catch (...) {
        cudaFree(dmel);
        cudaFree(dmis);
        cudaFree(dacc);
        cudaFree(bits);
        cudaFree(dcount);
        throw;
    }
    cudaFree(dmel);
    cudaFree(dmis);
    cudaFree(dacc);
    cudaFree(bits);
    cudaFree(dcount);
    return out;
}

} // namespace exaca
