// B200 kernels and pool runtime for ExaCA's per-cycle cellular-automaton update.
//
// One CA cycle (src/runCA.cpp:290-341; src/CAupdate.cpp:67-728) is three kernels over a pool of
// domains:
//   begin (k_step_begin, or the tail of the previous k_neighbours): per domain, the device-side
//          termination check, cycle/epoch advance and nucleation of the sites whose time has come
//          (nuclei are pre-sorted by time, one cursor each).
//   k_grow: streams the 16-byte records of the active cells (shared compacted list): diagonal
//          growth from the host-built increment table, solidification of cells with no liquid
//          neighbour, and a 64-bit atomicMin claim (epoch, capturer index) on every liquid neighbour
//          the octahedron reaches. Liquid neighbours come from a per-cell mask kept up to date by
//          captures and nucleations; the 26 critical lengths are read only when the diagonal has
//          reached the cached minimum over the liquid neighbours.
//   k_capture / k_neighbours: per claimed cell: capture by the lowest-index claimant (new decentred
//          octahedron, 26 critical lengths), mask updates of its active neighbours, and for those
//          the solidification re-check.
// The claim rule reproduces the Kokkos-Serial loop order exactly: serial visits active cells in
// ascending index and captures flip Liquid to Active in place, so the capturer of a cell is the
// lowest-index claimant, and an active cell sees a neighbour as liquid iff it was liquid at the
// start of the cycle and no lower-index cell claimed it. Only cells next to a claimed cell can lose
// their last such neighbour, so only they are re-checked.
//
// Arithmetic follows the reference's types and operation order; this file is compiled with
// -fmad=false so no multiply-add is contracted, and sqrt/division are IEEE round-to-nearest.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <sstream>
#include <stdexcept>

#include "pool.hpp"

namespace exaca {

#define CUDA_OK(x)                                                                                                     \
    do {                                                                                                               \
        cudaError_t e__ = (x);                                                                                         \
        if (e__ != cudaSuccess)                                                                                        \
            throw DeviceError(std::string("CUDA error ") + cudaGetErrorString(e__) + " at " #x);                     \
    } while (0)

__constant__ int c_nx[26];
__constant__ int c_ny[26];
__constant__ int c_nz[26];
// ItList (src/CAinitialize.cpp:676-745) as 26-bit direction masks per edge case, and the directions
// with a z component of +1 / -1
__constant__ unsigned int c_itmask[9];
__constant__ unsigned int c_zplus;
__constant__ unsigned int c_zminus;
// direction index of a neighbour offset (dz+1)*9 + (dx+1)*3 + (dy+1), and opposite directions
__constant__ int c_dir[27];
__constant__ int c_opp[26];

constexpr unsigned int kMaskFresh = 1u << 31; // liquid-neighbour mask not built yet
constexpr unsigned int kMaskDead = 1u << 30;  // solidified by a re-check: leaves the list next cycle
constexpr unsigned int kMaskKeep = 1u << 29;  // this cycle, a neighbour was captured by an index >= this cell's
constexpr unsigned int kDirBits = (1u << 26) - 1;
constexpr int kErrGrowthTable = 1;
constexpr int kErrListOverflow = 2;
constexpr int kErrBounds = 4;
constexpr int kBlock = 256;

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
    __shared__ unsigned int s_warp[kBlock / 32];
    __shared__ unsigned long long s_base;
    __shared__ int s_ok;
    const unsigned int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
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
        unsigned int v = lane < kBlock / 32 ? s_warp[lane] : 0;
        unsigned int inc2 = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            unsigned int u = __shfl_up_sync(0xffffffffu, inc2, o);
            if (lane >= (unsigned)o)
                inc2 += u;
        }
        if (lane < kBlock / 32)
            s_warp[lane] = inc2 - v;
        unsigned int total = __shfl_sync(0xffffffffu, inc2, kBlock / 32 - 1);
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
    __shared__ unsigned long long s_a[kBlock / 32], s_b[kBlock / 32];
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

// Edge case of src/CAfunctions.cpp:169-213 as a direction mask, restricted to the active window in
// z (src/CAupdate.cpp:328 checks MyNeighborZ < nzActive; the lower bound never binds for active
// cells and is kept as a guard).
__device__ __forceinline__ unsigned int neighbour_mask(const DomainDesc &D, int rx, int ry, int rz) {
    int b = (ry == 0) ? (rx == 0 ? 5 : (rx == D.mx - 1 ? 6 : 1))
                      : (ry == D.my - 1 ? (rx == 0 ? 7 : (rx == D.mx - 1 ? 8 : 2))
                                        : (rx == 0 ? 3 : (rx == D.mx - 1 ? 4 : 0)));
    unsigned int m = c_itmask[b];
    if (rz + 1 >= D.nz_active)
        m &= ~c_zplus;
    if (rz - 1 < 0)
        m &= ~c_zminus;
    return m;
}

__device__ __forceinline__ int nb_offset(int l, int plane, int my) { return c_nz[l] * plane + c_nx[l] * my + c_ny[l]; }

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
    D.lmask[c] = kMaskFresh;
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
// Warp-cooperative: every lane evaluates the (identical) geometry in lock step, then lane n < 26
// computes critical length n; lane 0 writes the scalar state. Returns the new DiagonalLength.
__device__ float capture_cell(const DomainDesc &D, unsigned int c, unsigned int t, int l, int lane) {
    // all loads first: capturer state, then its orientation
    const int h = D.gid[c];
    const float docx = D.doc[3ull * c + 0], docy = D.doc[3ull * c + 1], docz = D.doc[3ull * c + 2];
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
    double xp = GlobalX + c_nx[l] + 0.5;
    double yp = GlobalY + c_ny[l] + 0.5;
    double zp = GlobalZ + c_nz[l] + 0.5;
    double x0 = xp - cxold;
    double y0 = yp - cyold;
    double z0 = zp - czold;
    double mag0 = sqrtf((float)(x0 * x0 + y0 * y0 + z0 * z0));
    double Angle1 = (g0 * x0 + g1 * y0 + g2 * z0) / mag0;
    double Angle2 = (g3 * x0 + g4 * y0 + g5 * z0) / mag0;
    double Angle3 = (g6 * x0 + g7 * y0 + g8 * z0) / mag0;
    float s1 = (float)(2 * (Angle1 < 0) - 1);
    float s2 = (float)(2 * (Angle2 < 0) - 1);
    float s3 = (float)(2 * (Angle3 < 0) - 1);
    double Diag1X = g0 * s1, Diag1Y = g1 * s1, Diag1Z = g2 * s1;
    double Diag2X = g3 * s2, Diag2Y = g4 * s2, Diag2Z = g5 * s2;
    double Diag3X = g6 * s3, Diag3Y = g7 * s3, Diag3Z = g8 * s3;
    double U1x = Diag2X - Diag1X, U1y = Diag2Y - Diag1Y, U1z = Diag2Z - Diag1Z;
    double U2x = Diag3X - Diag1X, U2y = Diag3Y - Diag1Y, U2z = Diag3Z - Diag1Z;
    double UUx = U1y * U2z - U1z * U2y;
    double UUy = U1z * U2x - U1x * U2z;
    double UUz = U1x * U2y - U1y * U2x;
    double NDem = sqrtf((float)(UUx * UUx + UUy * UUy + UUz * UUz));
    double n0 = UUx / NDem, n1 = UUy / NDem, n2 = UUz / NDem;
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
    double Dist[3];
#pragma unroll
    for (int q = 0; q < 3; q++)
        Dist[q] = sqrtf((float)(((TX[q] - xp) * (TX[q] - xp)) + ((TY[q] - yp) * (TY[q] - yp)) +
                                ((TZ[q] - zp) * (TZ[q] - zp))));
    int x = (Dist[0] < Dist[1]);
    int y = (Dist[1] < Dist[2]);
    int z = (Dist[2] < Dist[0]);
    int idx = 2 * (z - y) * z + (y - x) * y;
    double mindist = Dist[idx];
    double xc = TX[idx], yc = TY[idx], zc = TZ[idx];
    int i1 = (idx + 1) % 3, i2 = (idx + 2) % 3;
    double x1 = TX[i1], y1 = TY[i1], z1 = TZ[i1];
    double x2 = TX[i2], y2 = TY[i2], z2 = TZ[i2];
    double D1 = sqrtf((float)(((xp - x2) * (xp - x2)) + ((yp - y2) * (yp - y2)) + ((zp - z2) * (zp - z2))));
    double D2 = sqrtf((float)(((xc - x2) * (xc - x2)) + ((yc - y2) * (yc - y2)) + ((zc - z2) * (zc - z2))));
    double D3 = sqrtf((float)(((xp - x1) * (xp - x1)) + ((yp - y1) * (yp - y1)) + ((zp - z1) * (zp - z1))));
    double D4 = sqrtf((float)(((xc - x1) * (xc - x1)) + ((yc - y1) * (yc - y1)) + ((zc - z1) * (zc - z1))));
    double I1 = 0, I2 = D2, J1 = 0, J2 = D4;
    if (mindist != 0) {
        I1 = D1 * ((xp - x2) * (xc - x2) + (yp - y2) * (yc - y2) + (zp - z2) * (zc - z2)) / (D1 * D2);
        I2 = D2 - I1;
        J1 = D3 * ((xp - x1) * (xc - x1) + (yp - y1) * (yc - y1) + (zp - z1) * (zc - z1)) / (D3 * D4);
        J2 = D4 - J1;
    }
    const double sqrt3 = sqrt(3.0);
    double L12 = 0.5 * (dmin(I1, sqrt3) + dmin(I2, sqrt3));
    double L13 = 0.5 * (dmin(J1, sqrt3) + dmin(J2, sqrt3));
    double NewODiagL = sqrt(2.0) * dmax(L12, L13);
    double cd0 = xc - cxold, cd1 = yc - cyold, cd2 = zc - czold;
    double nd = sqrt(cd0 * cd0 + cd1 * cd1 + cd2 * cd2);
    double uv0 = cd0 / nd, uv1 = cd1 / nd, uv2 = cd2 / nd;
    double cx = xc - NewODiagL * uv0;
    double cy = yc - NewODiagL * uv1;
    double cz = zc - NewODiagL * uv2;
    if (lane == 0) {
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
    if (lane < 26) {
        const int n = lane;
        double a0 = xp + c_nx[n] - cx;
        double b0 = yp + c_ny[n] - cy;
        double d0 = zp + c_nz[n] - cz;
        double q0 = a0 * Fx[0] + b0 * Fy[0] + d0 * Fz[0];
        double q1 = a0 * Fx[1] + b0 * Fy[1] + d0 * Fz[1];
        double q2 = a0 * Fx[2] + b0 * Fy[2] + d0 * Fz[2];
        double q3 = a0 * Fx[3] + b0 * Fy[3] + d0 * Fz[3];
        double m = dmax(dmax(fabs(q0), fabs(q1)), dmax(fabs(q2), fabs(q3)));
        D.cdl[26ull * t + n] = (float)m;
    }
    return (float)NewODiagL;
}

// A nucleation site stopped being liquid: its active neighbours drop it from their masks.
__device__ void drop_from_neighbour_masks(const DomainDesc &D, unsigned int t) {
    int rx, ry, rz;
    cell_coords(D, t, rx, ry, rz);
    const unsigned int valid = neighbour_mask(D, rx, ry, rz);
    const int plane = D.mx * D.my, my = D.my;
    for (unsigned int bits = valid; bits; bits &= bits - 1) {
        int l = __ffs(bits) - 1;
        unsigned int a = (unsigned int)((long long)t + nb_offset(l, plane, my));
        if (__ldcg(D.ctype + a) == kActive)
            atomicAnd(D.lmask + a, ~(1u << c_opp[l]));
    }
}

// ---------------------------------------------------------------------------------------------
// Start of a CA cycle for every domain (src/runCA.cpp:290-298, src/CAupdate.cpp:67-200), run by one
// block: list swap, device-side termination check, cycle advance, nucleation. Reads that may see
// data other blocks of the same kernel wrote go through L2 (__ldcg).
__device__ void begin_cycle(PoolState *P) {
    __shared__ int s_cur;
    if (threadIdx.x == 0) {
        // the list the previous cycle left becomes current; when it was a compacted copy, the old
        // one is emptied and carries no dropped records any more
        int prev = P->cur;
        int cur = P->pending;
        if (cur != prev) {
            P->cnt[prev] = 0;
            P->tombs = 0;
        }
        P->cur = cur;
        // compact when dropped records exceed an eighth of the list
        int compact = P->tombs * 8 > P->cnt[cur] ? 1 : 0;
        P->compact = compact;
        P->pending = compact ? cur ^ 1 : cur;
        if (compact)
            P->cnt[cur ^ 1] = 0;
        P->tcnt = 0;
        P->qcnt = 0;
        s_cur = cur;
    }
    __syncthreads();
    const int cur = s_cur;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    unsigned long long nucleated = 0;
    for (int d = warp; d < P->n_domains; d += nwarps) {
        DomainDesc &D = P->desc[d];
        if (D.ctype == nullptr || D.done)
            continue;
        if (D.check_mode && D.cycle > 0 && D.cycle % 1000 == 0 && domain_liquid(D) == 0) {
            // src/CAupdate.cpp:782-783: no superheated or undercooled liquid left
            if (lane == 0)
                D.done = 1;
            continue;
        }
        const int cycle = D.cycle + 1;
        __syncwarp();
        if (lane == 0) {
            D.cycle = cycle;
            D.epoch = D.epoch + 1;
        }
        // src/CAupdate.cpp:76-198: sites with cycle >= NucleationTimes that are still liquid
        int cursor = D.nuc_cursor;
        int fired_total = 0;
        while (cursor < D.n_nuclei) {
            int idx = cursor + lane;
            int t = idx < D.n_nuclei ? D.nuc_time[idx] : INT_MAX;
            unsigned int due = __ballot_sync(0xffffffffu, t <= cycle);
            // nuclei are sorted by time, so the due ones form a prefix
            int n_due = __popc(due);
            bool fire = false;
            unsigned int loc = 0;
            if (t <= cycle) {
                int l = D.nuc_loc[idx];
                if (l < 0 || l >= D.active_size) {
                    atomicOr(&D.error, kErrBounds);
                }
                else {
                    loc = (unsigned int)l;
                    fire = __ldcg(D.ctype + loc) == kLiquid && D.layer[loc] <= 0;
                }
            }
            if (fire) {
                make_fresh_octahedron(D, loc);
                unsigned long long pos = warp_reserve(&P->cnt[cur], P->capacity, &P->error);
                if (pos != ULLONG_MAX) {
                    ActiveRec r;
                    r.cell = loc;
                    r.dl = 0.01f;
                    r.cdl_min = 0.0f;
                    r.cts = D.cts[loc];
                    P->rec[cur][pos] = r;
                    P->rdom[cur][pos] = (unsigned int)d;
                }
                D.ctype[loc] = kActive;
            }
            __syncwarp();
            if (fire)
                drop_from_neighbour_masks(D, loc);
            unsigned int fired = __ballot_sync(0xffffffffu, fire);
            fired_total += __popc(fired);
            cursor += n_due;
            if (n_due < 32)
                break;
        }
        if (lane == 0) {
            D.nuc_cursor = cursor;
            D.nn += fired_total;
            D.liquid -= fired_total;
            nucleated += fired_total;
        }
    }
    if (lane == 0 && nucleated)
        atomicAdd(&P->stat[0][kStatNucleated], nucleated);
}

__global__ void k_step_begin(PoolState *P) { begin_cycle(P); }

// ---------------------------------------------------------------------------------------------
// Per-cycle growth of the active cells, split by cost:
//   k_grow    streams every record (kBatch per thread, loads issued first): eligibility, diagonal
//             growth (src/CAupdate.cpp:257-261), drop of finished / re-check-solidified cells, and
//             solidification of cells whose liquid mask is empty. A record whose mask must still
//             be built, or whose diagonal reached the cached minimum critical length, is flagged
//             (cdl_min = kNeedsClaim) for
//   k_claim   one thread per flagged record, chunks handed out dynamically: the liquid mask from
//             the 26 neighbour types, the critical-length row (13 aligned 8-byte loads), and the
//             claims (src/CAupdate.cpp:320-352).
constexpr unsigned int kNeedsClaim = 0xffffffffu; // NaN pattern in ActiveRec::cdl_min
constexpr int kBatch = 4;

struct GrowStats {
    unsigned long long listed = 0, grown = 0, dropped = 0, flagged = 0;
};

// Growth step of one record with its liquid mask and growth increment loaded. Returns 0: drop
// the record, 1: keep it unchanged (not eligible yet), 2: keep the updated record.
__device__ __forceinline__ int grow_record(DomainDesc &D, ActiveRec &r, unsigned int m, double inc, bool inc_ok,
                                           GrowStats &st) {
    const unsigned int c = r.cell;
    st.listed++;
    if (D.done || (m & kMaskDead)) {
        // finished domain, or solidified by last cycle's re-check
        D.dl[c] = r.dl;
        return 0;
    }
    if (!(D.cycle > r.cts))
        return 1; // single-layer problems only: LayerID <= layer always holds
    st.grown++;
    if (!inc_ok)
        atomicOr(&D.error, kErrGrowthTable);
    const float dl = (float)((double)r.dl + inc);
    r.dl = dl;
    if ((m & kMaskFresh) || dl >= r.cdl_min) {
        r.cdl_min = __uint_as_float(kNeedsClaim);
        st.flagged++;
        return 2;
    }
    if (m == 0) {
        // no liquid neighbour: LCount stays 0 (src/CAupdate.cpp:722-725)
        D.ctype[c] = kSolid;
        D.dl[c] = dl;
        return 0;
    }
    return 2;
}

__device__ __forceinline__ void load_growth(const DomainDesc &D, const ActiveRec &r, unsigned int &m, double &inc,
                                            bool &ok) {
    m = D.lmask[r.cell];
    if (m & kMaskKeep) {
        // the neighbour verdict of the previous cycle does not carry over
        m &= ~kMaskKeep;
        D.lmask[r.cell] = m;
    }
    // undercooling after the executed updates since the liquidus (src/CAupdate.cpp:236-237)
    long long nu = executed_upto(D, D.cycle) - executed_upto(D, r.cts);
    if (D.zero_du && D.du[r.cell] == 0.0f)
        nu = 0;
    ok = nu >= 0 && nu < D.growth_len;
    inc = (ok && D.cycle > r.cts) ? __ldg(D.growth + nu) : 0.0;
}

__global__ void __launch_bounds__(kBlock) k_grow(PoolState *P) {
    const int cur = P->cur;
    const unsigned long long n = P->cnt[cur];
    ActiveRec *in = P->rec[cur];
    const unsigned int *in_dom = P->rdom[cur];
    DomainDesc *desc = P->desc;
    GrowStats st;
    if (!P->compact) {
        // records are updated in place; dropped ones become tombstones
        const unsigned long long step = (unsigned long long)gridDim.x * kBlock * kBatch;
        // block-uniform loop: block_reserve_on is reached by every thread
        for (unsigned long long b0 = (unsigned long long)blockIdx.x * kBlock * kBatch; b0 < n; b0 += step) {
            const unsigned long long base = b0 + threadIdx.x;
            ActiveRec r[kBatch];
            unsigned int dom[kBatch], m[kBatch];
            double inc[kBatch];
            bool ok[kBatch];
#pragma unroll
            for (int q = 0; q < kBatch; q++) {
                const unsigned long long i = base + (unsigned long long)q * kBlock;
                r[q].cell = kTombstone;
                dom[q] = 0;
                if (i < n) {
                    r[q] = in[i];
                    dom[q] = in_dom[i];
                }
            }
#pragma unroll
            for (int q = 0; q < kBatch; q++) {
                m[q] = 0;
                inc[q] = 0.0;
                ok[q] = true;
                if (r[q].cell != kTombstone)
                    load_growth(desc[dom[q]], r[q], m[q], inc[q], ok[q]);
            }
            unsigned int flagged = 0;
#pragma unroll
            for (int q = 0; q < kBatch; q++) {
                if (r[q].cell == kTombstone)
                    continue;
                const unsigned long long i = base + (unsigned long long)q * kBlock;
                const int a = grow_record(desc[dom[q]], r[q], m[q], inc[q], ok[q], st);
                if (a == 0) {
                    ActiveRec tomb = r[q];
                    tomb.cell = kTombstone;
                    tomb.cdl_min = 0.0f;
                    in[i] = tomb;
                    st.dropped++;
                }
                else if (a == 2) {
                    *reinterpret_cast<float2 *>(&in[i].dl) = make_float2(r[q].dl, r[q].cdl_min);
                    if (__float_as_uint(r[q].cdl_min) == kNeedsClaim)
                        flagged |= 1u << q;
                }
            }
            const unsigned long long qpos = block_reserve_on(&P->qcnt, P->capacity, &P->error, __popc(flagged));
            if (qpos != ULLONG_MAX) {
                unsigned long long k = qpos;
#pragma unroll
                for (int q = 0; q < kBatch; q++)
                    if (flagged & (1u << q))
                        P->queue[k++] = (unsigned int)(base + (unsigned long long)q * kBlock);
            }
        }
    }
    else {
        // compaction: the survivors are written to the other list
        const int nxt = cur ^ 1;
        ActiveRec *out = P->rec[nxt];
        unsigned int *out_dom = P->rdom[nxt];
        const unsigned long long stride = (unsigned long long)gridDim.x * kBlock;
        // block-uniform loop: block_reserve is reached by every thread
        for (unsigned long long i0 = (unsigned long long)blockIdx.x * kBlock; i0 < n; i0 += stride) {
            const unsigned long long i = i0 + threadIdx.x;
            bool keep = false;
            ActiveRec r;
            unsigned int dom = 0;
            if (i < n) {
                r = in[i];
                dom = in_dom[i];
                if (r.cell != kTombstone) {
                    unsigned int m;
                    double inc;
                    bool ok;
                    load_growth(desc[dom], r, m, inc, ok);
                    keep = grow_record(desc[dom], r, m, inc, ok, st) != 0;
                }
            }
            const unsigned long long pos = block_reserve(P, nxt, keep ? 1u : 0u);
            const bool flag = keep && pos != ULLONG_MAX && __float_as_uint(r.cdl_min) == kNeedsClaim;
            if (keep && pos != ULLONG_MAX) {
                out[pos] = r;
                out_dom[pos] = dom;
            }
            const unsigned long long qpos = block_reserve_on(&P->qcnt, P->capacity, &P->error, flag ? 1u : 0u);
            if (flag && qpos != ULLONG_MAX)
                P->queue[qpos] = (unsigned int)pos;
        }
    }
    block_stats(P, st.listed, st.grown, kStatListed, kStatGrown);
    block_stats(P, st.dropped, st.flagged, kStatDropped, kStatFlagged);
    if (!P->compact) {
        // dropped records stay as tombstones until the next compaction
        __shared__ unsigned long long s_d;
        if (threadIdx.x == 0)
            s_d = 0;
        __syncthreads();
        if (st.dropped)
            atomicAdd(&s_d, st.dropped);
        __syncthreads();
        if (threadIdx.x == 0 && s_d)
            atomicAdd(&P->tombs, s_d);
    }
}

__global__ void __launch_bounds__(kBlock) k_claim(PoolState *P) {
    const int lst = P->pending; // the list the growth pass just wrote
    const unsigned long long nq = P->qcnt;
    ActiveRec *recs = P->rec[lst];
    const unsigned int *rdom = P->rdom[lst];
    DomainDesc *desc = P->desc;
    unsigned long long st_claims = 0, st_rows = 0, st_fresh = 0, st_dropped = 0;
    const unsigned long long nthreads = (unsigned long long)gridDim.x * kBlock;
    const unsigned long long me = (unsigned long long)threadIdx.x * gridDim.x + blockIdx.x;
    // block-uniform loop (block_reserve_on); consecutive items on different blocks
    for (unsigned long long q0 = 0; q0 < nq; q0 += nthreads) {
        const unsigned long long qi = q0 + me;
        unsigned int first = 0, pushed_dom = 0;
        unsigned int pushed_cell = 0;
        int first_plane = 0, first_my = 0;
        do {
        if (qi >= nq)
            break;
        const unsigned long long i = P->queue[qi];
        const ActiveRec rec = recs[i];
        if (rec.cell == kTombstone || __float_as_uint(rec.cdl_min) != kNeedsClaim)
            continue;
        const unsigned int c = rec.cell;
        const unsigned int dom = rdom[i];
        DomainDesc &D = desc[dom];
        const float dl = rec.dl;
        const int plane = D.mx * D.my, my = D.my;
        int rx, ry, rz;
        cell_coords(D, c, rx, ry, rz);
        unsigned int m = D.lmask[c];
        if (m & kMaskFresh) {
            // liquid neighbours from the 26 neighbour types (src/CAupdate.cpp:320-334); no other
            // thread writes this cell's mask now, captures and nucleations clear bits later
            st_fresh++;
            const unsigned int valid = neighbour_mask(D, rx, ry, rz);
            const int8_t *ct = D.ctype + c;
            m = 0;
#pragma unroll
            for (int l = 0; l < 26; l++)
                if ((valid & (1u << l)) && ct[nb_offset(l, plane, my)] == kLiquid)
                    m |= 1u << l;
            D.lmask[c] = m;
        }
        if (m == 0) {
            // no liquid neighbour: LCount stays 0 (src/CAupdate.cpp:722-725)
            D.ctype[c] = kSolid;
            D.dl[c] = dl;
            ActiveRec tomb = rec;
            tomb.cell = kTombstone;
            tomb.cdl_min = 0.0f;
            recs[i] = tomb;
            st_dropped++;
            continue;
        }
        // the 26 critical lengths as 13 aligned 8-byte loads (26 * 4 * c is 8-byte aligned)
        st_rows++;
        const float2 *row = reinterpret_cast<const float2 *>(D.cdl + 26ull * c);
        float cdl[26];
#pragma unroll
        for (int q = 0; q < 13; q++) {
            float2 v = row[q];
            cdl[2 * q] = v.x;
            cdl[2 * q + 1] = v.y;
        }
        float nm = __int_as_float(0x7f800000);
        unsigned int reach = 0;
#pragma unroll
        for (int l = 0; l < 26; l++) {
            if (m & (1u << l)) {
                nm = (cdl[l] < nm) ? cdl[l] : nm;
                if (dl >= cdl[l])
                    reach |= 1u << l;
            }
        }
        recs[i].cdl_min = nm;
        if (reach) {
            // claims (src/CAupdate.cpp:336-352): lowest index wins; the first claimant of a cell in
            // this cycle lists it for k_capture / k_neighbours
            const unsigned long long key = ((unsigned long long)(0xffffffffu - D.epoch) << 32) | (unsigned long long)c;
            const unsigned int want = 0xffffffffu - D.epoch;
#pragma unroll
            for (int l = 0; l < 26; l++) {
                if (reach & (1u << l)) {
                    unsigned long long old = atomicMin(D.claim + (long long)c + nb_offset(l, plane, my), key);
                    if ((unsigned int)(old >> 32) != want)
                        first |= 1u << l;
                }
            }
            st_claims += __popc(reach);
            pushed_dom = dom;
            pushed_cell = c;
            first_plane = plane;
            first_my = my;
        }
        } while (false);
        // list the cells this thread claimed first (block-aggregated reservation)
        const unsigned long long pos = block_reserve_on(&P->tcnt, P->capacity, &P->error, __popc(first));
        if (pos != ULLONG_MAX) {
            unsigned long long k = pos;
            for (unsigned int bits = first; bits; bits &= bits - 1) {
                int l = __ffs(bits) - 1;
                P->tgt[k++] = ((unsigned long long)pushed_dom << 32) |
                              (unsigned int)((long long)pushed_cell + nb_offset(l, first_plane, first_my));
            }
        }
    }
    block_stats(P, st_claims, st_rows, kStatClaims, kStatRowReads);
    block_stats(P, st_fresh, 0, kStatFresh, kStatFresh);
    if (st_dropped && !P->compact)
        atomicAdd(&P->tombs, st_dropped);
}

// Every cell claimed this cycle is captured by its lowest-index claimant (src/CAupdate.cpp:336-563,
// 713-717). Two independent passes over the claimed cells:
//   k_capture     one thread per claimed cell: the new octahedron, 26 critical lengths, GrainID,
//                 and its record in the next cycle's list.
//   k_neighbours  26 threads per claimed cell: each active neighbour drops the cell from its liquid
//                 mask, and a neighbour grown this cycle re-checks whether it still sees a liquid
//                 cell (src/CAupdate.cpp:722-725). With kTail the last block to finish starts the
//                 next cycle.
// Neither pass reads what the other writes: the re-check uses the claims and the unclaimed mask
// bits only, and a cell being captured still has its initial (not yet built) mask.
__global__ void __launch_bounds__(kBlock) k_capture(PoolState *P) {
    const int app = P->pending; // list of the next cycle
    const unsigned long long T = P->tcnt;
    // claimed cell j gets record slot base + j (the count grows by T in k_neighbours)
    const unsigned long long base = P->cnt[app];
    if (base + T > P->capacity) {
        if (threadIdx.x == 0 && blockIdx.x == 0)
            atomicOr(&P->error, kErrListOverflow);
        return;
    }
    DomainDesc *desc = P->desc;
    const int lane = threadIdx.x & 31;
    // one warp per claimed cell, consecutive cells on different blocks (spread over all SMs)
    const unsigned long long nwarps = (unsigned long long)gridDim.x * (kBlock / 32);
    const unsigned long long w0 = (unsigned long long)(threadIdx.x >> 5) * gridDim.x + blockIdx.x;
    unsigned long long st_cap = 0;
    for (unsigned long long j = w0; j < T; j += nwarps) {
        const unsigned long long e = P->tgt[j];
        const unsigned int dom = (unsigned int)(e >> 32);
        const unsigned int t = (unsigned int)e;
        DomainDesc &D = desc[dom];
        const unsigned int w = (unsigned int)__ldcg(D.claim + t);
        const int cts_t = __ldg(D.cts + t);
        int wx, wy, wz, tx, ty, tz;
        cell_coords(D, w, wx, wy, wz);
        cell_coords(D, t, tx, ty, tz);
        const int l = c_dir[(tz - wz + 1) * 9 + (tx - wx + 1) * 3 + (ty - wy + 1)];
        const float new_dl = capture_cell(D, w, t, l, lane);
        __syncwarp();
        if (lane == 0) {
            D.lmask[t] = kMaskFresh;
            ActiveRec r;
            r.cell = t;
            r.dl = new_dl;
            r.cdl_min = 0.0f;
            r.cts = cts_t;
            P->rec[app][base + j] = r;
            P->rdom[app][base + j] = dom;
            // read as active only from the next kernel on, after the octahedron data is written
            D.ctype[t] = kActive;
            atomicAdd((unsigned long long *)&D.liquid_shard[(blockIdx.x + j) & (kLiquidShards - 1)],
                      (unsigned long long)(-1ll));
            st_cap++;
        }
    }
    block_stats(P, st_cap, 0, kStatCaptured, kStatCaptured);
}

template <bool kTail> __global__ void __launch_bounds__(kBlock) k_neighbours(PoolState *P) {
    const unsigned long long n = P->tcnt * 26ull;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        // the records k_capture wrote at fixed slots join the next cycle's list
        const int app = P->pending;
        if (P->cnt[app] + P->tcnt <= P->capacity)
            P->cnt[app] += P->tcnt;
    }
    DomainDesc *desc = P->desc;
    unsigned long long st_rc = 0;
    // consecutive items on different blocks (spread over all SMs)
    const unsigned long long nthreads = (unsigned long long)gridDim.x * kBlock;
    for (unsigned long long j = (unsigned long long)threadIdx.x * gridDim.x + blockIdx.x; j < n; j += nthreads) {
        const unsigned long long q = j / 26ull;
        const int l = (int)(j - q * 26ull);
        const unsigned long long e = P->tgt[q];
        const unsigned int dom = (unsigned int)(e >> 32);
        const unsigned int t = (unsigned int)e;
        DomainDesc &D = desc[dom];
        int tx, ty, tz;
        cell_coords(D, t, tx, ty, tz);
        if (!(neighbour_mask(D, tx, ty, tz) & (1u << l)))
            continue;
        const unsigned int a = (unsigned int)((long long)t + nb_offset(l, D.mx * D.my, D.my));
        const unsigned int w = (unsigned int)__ldcg(D.claim + t);
        if (__ldcg(D.ctype + a) != kActive)
            continue;
        // Serial order (src/CAupdate.cpp:333-334, 722-725): active cell a saw the captured cell t
        // as liquid iff t's capturer w does not precede a. a keeps a liquid neighbour iff it has an
        // unclaimed one (a set mask bit that nobody clears) or a claimed one with w >= a. Every
        // claimed liquid neighbour clears its own bit exactly once, so the update that clears the
        // last direction bit sees the final verdict: KEEP is always set before the clear of the
        // same update, and an update's two atomics reach the word in program order.
        if (w >= a)
            atomicOr(D.lmask + a, kMaskKeep);
        const unsigned int bit = 1u << c_opp[l];
        const unsigned int old = atomicAnd(D.lmask + a, ~bit);
        if ((old & (kMaskFresh | kMaskDead)) || (old & kDirBits) != bit || (old & kMaskKeep))
            continue;
        // a lost its last liquid neighbour; it solidifies if it was grown this cycle
        if (D.cycle > __ldg(D.cts + a)) {
            st_rc++;
            D.ctype[a] = kSolid;
            atomicOr(D.lmask + a, kMaskDead);
        }
    }
    block_stats(P, st_rc, 0, kStatRechecks, kStatRechecks);
    if (kTail) {
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
            begin_cycle(P);
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Census of src/CAupdate.cpp:738-808 for one domain (layer 0 is the only layer).
__global__ void k_census(const DomainDesc *Dp, Census *out) {
    const DomainDesc &D = *Dp;
    unsigned long long a[5] = {0, 0, 0, 0, 0};
    unsigned long long mn = ULLONG_MAX;
    const long long stride = (long long)gridDim.x * blockDim.x;
    int cycle = D.cycle;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < D.domain_size; c += stride) {
        int t = D.ctype[c];
        int ly = D.layer[c];
        int cts = D.cts[c];
        if (ly == 0) {
            if (t == kLiquid) {
                if (cts > cycle)
                    a[0]++;
                else
                    a[1]++;
                if (c < D.active_size && (unsigned long long)cts < mn)
                    mn = (unsigned long long)(long long)cts;
            }
            else if (t == kActive)
                a[2]++;
            else if (t == kSolid)
                a[3]++;
        }
        else if (t == kLiquid) {
            a[4]++;
        }
    }
    for (int q = 0; q < 5; q++) {
        unsigned long long v = a[q];
        for (int o = 16; o; o >>= 1)
            v += __shfl_down_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0 && v)
            atomicAdd((unsigned long long *)out + q, v);
    }
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

// Initially active cells: fresh octahedra and the first records (src/CAinitialize.cpp:1929-2044).
__global__ void k_init_active(PoolState *P, int dom, int list_slot) {
    DomainDesc &D = P->desc[dom];
    long long plane = (long long)D.mx * D.my;
    long long lo = plane, hi = plane * (D.nz - 1);
    long long zmax = plane * ((long long)D.zbound_high + 1);
    if (hi > zmax)
        hi = zmax;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long c0 = lo + (long long)blockIdx.x * blockDim.x; c0 < hi; c0 += stride) {
        long long c = c0 + threadIdx.x;
        bool act = c < hi && D.ctype[c] == kActive;
        if (act)
            make_fresh_octahedron(D, (unsigned int)c);
        bool listed = act && c < D.active_size;
        unsigned long long pos = block_reserve(P, list_slot, listed ? 1u : 0u);
        if (listed && pos != ULLONG_MAX) {
            ActiveRec r;
            r.cell = (unsigned int)c;
            r.dl = 0.01f;
            r.cdl_min = 0.0f;
            r.cts = D.cts[c];
            P->rec[list_slot][pos] = r;
            P->rdom[list_slot][pos] = (unsigned int)dom;
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
        const DomainDesc &D = P->desc[P->rdom[nxt][i]];
        if (r.cell != kTombstone && D.dl)
            D.dl[r.cell] = r.dl;
    }
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
} // namespace

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

size_t Pool::slot_bytes(const Problem &p) {
    size_t N = (size_t)p.g.domain_size, A = (size_t)p.g.active_size;
    return N * (1 + 4 + 4 + 1 + 4) + A * (4 + 12 + 104 + 8 + 4) + p.nuclei_loc.size() * 8 + 64 * 1024;
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
    int it[9][26], lens[9];
    build_itlist(it, lens);
    CUDA_OK(cudaMemcpyToSymbol(c_nx, kNeighborX, sizeof(kNeighborX)));
    CUDA_OK(cudaMemcpyToSymbol(c_ny, kNeighborY, sizeof(kNeighborY)));
    CUDA_OK(cudaMemcpyToSymbol(c_nz, kNeighborZ, sizeof(kNeighborZ)));
    unsigned int itmask[9], zplus = 0, zminus = 0;
    for (int b = 0; b < 9; b++) {
        itmask[b] = 0;
        for (int q = 0; q < lens[b]; q++)
            itmask[b] |= 1u << it[b][q];
    }
    for (int l = 0; l < 26; l++) {
        if (kNeighborZ[l] == 1)
            zplus |= 1u << l;
        if (kNeighborZ[l] == -1)
            zminus |= 1u << l;
    }
    int dir[27], opp[26];
    for (int q = 0; q < 27; q++)
        dir[q] = -1;
    for (int l = 0; l < 26; l++)
        dir[(kNeighborZ[l] + 1) * 9 + (kNeighborX[l] + 1) * 3 + (kNeighborY[l] + 1)] = l;
    for (int l = 0; l < 26; l++)
        opp[l] = dir[(1 - kNeighborZ[l]) * 9 + (1 - kNeighborX[l]) * 3 + (1 - kNeighborY[l])];
    CUDA_OK(cudaMemcpyToSymbol(c_dir, dir, sizeof(dir)));
    CUDA_OK(cudaMemcpyToSymbol(c_opp, opp, sizeof(opp)));
    CUDA_OK(cudaMemcpyToSymbol(c_itmask, itmask, sizeof(itmask)));
    CUDA_OK(cudaMemcpyToSymbol(c_zplus, &zplus, sizeof(zplus)));
    CUDA_OK(cudaMemcpyToSymbol(c_zminus, &zminus, sizeof(zminus)));
    max_domains_ = 8192;
    capacity_ = std::max<unsigned long long>(list_capacity, 1024);
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
    }
    CUDA_OK(cudaMalloc(&ps.tgt, capacity_ * sizeof(unsigned long long)));
    CUDA_OK(cudaMalloc(&ps.queue, capacity_ * sizeof(unsigned int)));
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
            }
            cudaFree(ps.tgt);
            cudaFree(ps.queue);
        }
        cudaFree(dstate_);
    }
    cudaFree(ddesc_);
    cudaFree(census_buf_);
    cudaStreamDestroy(S(stream_));
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
    return tables_[p.cfg.orientation_file] = t;
}

void Pool::push_desc(int slot) {
    CUDA_OK(cudaMemcpyAsync(ddesc_ + slot, &host_desc_[slot], sizeof(DomainDesc), cudaMemcpyHostToDevice, S(stream_)));
    CUDA_OK(cudaStreamSynchronize(S(stream_)));
}

void Pool::ensure_growth(int slot, long long needed) {
    SlotHost &s = slots_[slot];
    if (needed < s.growth_len)
        return;
    long long len = std::max<long long>(needed + 1, std::max<long long>(2LL * s.growth_len, 4096));
    if (len > INT_MAX / 2)
        throw Unsupported("growth table too long");
    std::vector<double> g;
    build_growth_table(*s.problem, (int)len, g);
    double *d = nullptr;
    CUDA_OK(cudaMalloc(&d, len * sizeof(double)));
    CUDA_OK(cudaMemcpy(d, g.data(), len * sizeof(double), cudaMemcpyHostToDevice));
    CUDA_OK(cudaStreamSynchronize(S(stream_)));
    if (s.growth)
        CUDA_OK(cudaFree(s.growth));
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
    CUDA_OK(cudaStreamSynchronize(S(stream_)));
}

int Pool::admit(std::shared_ptr<const Problem> pp, int check_mode) {
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
    size_t N = g.domain_size, A = g.active_size;
    DomainDesc d;
    std::memset(&d, 0, sizeof(d));
    d.ctype = dalloc<int8_t>(N, s.allocs, s.bytes);
    d.gid = dalloc<int32_t>(N, s.allocs, s.bytes);
    d.cts = dalloc<int32_t>(N, s.allocs, s.bytes);
    d.layer = dalloc<int8_t>(N, s.allocs, s.bytes);
    d.du = dalloc<float>(N, s.allocs, s.bytes);
    d.dl = dalloc<float>(A, s.allocs, s.bytes);
    d.doc = dalloc<float>(3 * A, s.allocs, s.bytes);
    d.cdl = dalloc<float>(26 * A, s.allocs, s.bytes);
    d.claim = dalloc<unsigned long long>(A, s.allocs, s.bytes);
    d.lmask = dalloc<unsigned int>(A, s.allocs, s.bytes);
    // nuclei in time order; ties keep the reference's order (order does not change results)
    size_t P = p.nuclei_loc.size();
    std::vector<int> order(P);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return p.nuclei_time[a] < p.nuclei_time[b]; });
    std::vector<int32_t> nl(P), nt(P);
    for (size_t q = 0; q < P; q++) {
        nl[q] = p.nuclei_loc[order[q]];
        nt[q] = p.nuclei_time[order[q]];
    }
    int32_t *dnl = dalloc<int32_t>(P, s.allocs, s.bytes);
    int32_t *dnt = dalloc<int32_t>(P, s.allocs, s.bytes);
    cudaStream_t st = S(stream_);
    CUDA_OK(cudaMemcpyAsync(d.ctype, p.cell_type.data(), N, cudaMemcpyHostToDevice, st));
    CUDA_OK(cudaMemcpyAsync(d.gid, p.grain_id.data(), N * 4, cudaMemcpyHostToDevice, st));
    CUDA_OK(cudaMemcpyAsync(d.cts, p.cts.data(), N * 4, cudaMemcpyHostToDevice, st));
    CUDA_OK(cudaMemcpyAsync(d.layer, p.layer_id.data(), N, cudaMemcpyHostToDevice, st));
    CUDA_OK(cudaMemcpyAsync(d.du, p.du.data(), N * 4, cudaMemcpyHostToDevice, st));
    CUDA_OK(cudaMemsetAsync(d.dl, 0, A * 4, st));
    CUDA_OK(cudaMemsetAsync(d.claim, 0xff, A * 8, st));
    CUDA_OK(cudaMemsetAsync(d.lmask, 0x80, A * 4, st)); // kMaskFresh in every cell
    if (P) {
        CUDA_OK(cudaMemcpyAsync(dnl, nl.data(), P * 4, cudaMemcpyHostToDevice, st));
        CUDA_OK(cudaMemcpyAsync(dnt, nt.data(), P * 4, cudaMemcpyHostToDevice, st));
    }
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
    d.check_mode = check_mode;
    d.domain_size = g.domain_size;
    d.active_size = g.active_size;
    d.du_value = p.du_value;
    long long liquid = 0;
    int zero_du = 0;
    for (long i = 0; i < g.domain_size; i++) {
        int8_t t = p.cell_type[i];
        if (t == kLiquid && p.layer_id[i] == 0)
            liquid++;
        if ((t == kLiquid || t == kActive) && p.du[i] == 0.0f)
            zero_du = 1;
    }
    d.liquid = liquid;
    d.zero_du = zero_du;
    host_desc_[slot] = d;
    push_desc(slot);
    ensure_growth(slot, 4096);
    if (!p.voronoi_seeds.empty() || p.cfg.simulation_type == "S") {
        int nseeds = (int)(p.voronoi_seeds.size() / 3);
        int32_t *dseeds = nullptr;
        if (nseeds) {
            CUDA_OK(cudaMalloc(&dseeds, p.voronoi_seeds.size() * 4));
            CUDA_OK(cudaMemcpyAsync(dseeds, p.voronoi_seeds.data(), p.voronoi_seeds.size() * 4,
                                    cudaMemcpyHostToDevice, st));
        }
        long long blocks = (g.domain_size + 255) / 256;
        k_voronoi<<<(unsigned)blocks, 256, 3 * 1024 * sizeof(int), st>>>(ddesc_ + slot, dseeds, nseeds,
                                                                         (float)(g.active_size));
        CUDA_OK(cudaGetLastError());
        CUDA_OK(cudaStreamSynchronize(st));
        if (dseeds)
            CUDA_OK(cudaFree(dseeds));
    }
    // register the domain, then build its initial active list in the list the next cycle consumes
    PoolState ps;
    CUDA_OK(cudaMemcpyAsync(&ps, dstate_, sizeof(ps), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    int n_domains = std::max(ps.n_domains, slot + 1);
    CUDA_OK(cudaMemcpyAsync((char *)dstate_ + offsetof(PoolState, n_domains), &n_domains, sizeof(int),
                            cudaMemcpyHostToDevice, st));
    int next_slot = ps.pending;
    k_init_active<<<num_sms_ * 4, 256, 0, st>>>(dstate_, slot, next_slot);
    CUDA_OK(cudaGetLastError());
    CUDA_OK(cudaStreamSynchronize(st));
    bytes_in_use_ += s.bytes;
    return slot;
}

void Pool::retire(int slot) {
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
    CUDA_OK(cudaStreamSynchronize(st));
    DomainDesc zero;
    std::memset(&zero, 0, sizeof(zero));
    zero.done = 1;
    host_desc_[slot] = zero;
    CUDA_OK(cudaMemcpyAsync(ddesc_ + slot, &zero, sizeof(zero), cudaMemcpyHostToDevice, st));
    CUDA_OK(cudaStreamSynchronize(st));
    for (void *p : s.allocs)
        CUDA_OK(cudaFree(p));
    if (s.growth)
        CUDA_OK(cudaFree(s.growth));
    bytes_in_use_ -= s.bytes;
    s = SlotHost();
}

void Pool::launch_step() {
    cudaStream_t st = S(stream_);
    if (grid_grow_ == 0) {
        // persistent grids: every resident block slot on the device, grid-stride over the list
        int b1 = 0, b2 = 0;
        int b3 = 0, b4 = 0;
        CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1, k_grow, kBlock, 0));
        CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b2, k_capture, kBlock, 0));
        CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b3, k_claim, kBlock, 0));
        CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b4, k_neighbours<true>, kBlock, 0));
        grid_grow_ = num_sms_ * std::max(b1, 1);
        grid_capture_ = num_sms_ * std::max(b2, 1);
        grid_claim_ = num_sms_ * std::max(b3, 1);
        grid_nb_ = num_sms_ * std::max(b4, 1);
    }
    k_step_begin<<<1, kBlock, 0, st>>>(dstate_);
    k_grow<<<grid_grow_, kBlock, 0, st>>>(dstate_);
    k_claim<<<grid_claim_, kBlock, 0, st>>>(dstate_);
    k_capture<<<grid_capture_, kBlock, 0, st>>>(dstate_);
    k_neighbours<false><<<grid_nb_, kBlock, 0, st>>>(dstate_);
    launches_ += 5;
}

// n cycles in one stream sequence: the begin of cycles 2..n runs in the tail of the previous
// capture kernel, so a cycle costs two launches.
void Pool::launch_cycles(int n) {
    if (n <= 0)
        return;
    if (grid_grow_ == 0)
        launch_step(), n--; // sizes the grids on first use
    if (n <= 0)
        return;
    cudaStream_t st = S(stream_);
    k_step_begin<<<1, kBlock, 0, st>>>(dstate_);
    launches_ += 1 + 4ull * n;
    for (int q = 0; q < n; q++) {
        k_grow<<<grid_grow_, kBlock, 0, st>>>(dstate_);
        k_claim<<<grid_claim_, kBlock, 0, st>>>(dstate_);
        k_capture<<<grid_capture_, kBlock, 0, st>>>(dstate_);
        if (q + 1 < n)
            k_neighbours<true><<<grid_nb_, kBlock, 0, st>>>(dstate_);
        else
            k_neighbours<false><<<grid_nb_, kBlock, 0, st>>>(dstate_);
    }
}

void Pool::build_graph() {
    if (graph_exec_)
        return;
    graph_steps_ = 50;
    cudaStream_t st = S(stream_);
    cudaGraph_t graph;
    if (grid_grow_ == 0)
        throw DeviceError("grids not sized before graph capture");
    CUDA_OK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    launch_cycles(graph_steps_);
    CUDA_OK(cudaStreamEndCapture(st, &graph));
    cudaGraphExec_t ex;
    CUDA_OK(cudaGraphInstantiate(&ex, graph, 0));
    CUDA_OK(cudaGraphDestroy(graph));
    graph_exec_ = ex;
}

void Pool::step(int n) {
    if (n <= 0)
        return;
    cycles_launched_ += (unsigned long long)n;
    CUDA_OK(cudaSetDevice(device_));
    for (int s = 0; s < (int)slots_.size(); s++) {
        if (!slots_[s].used)
            continue;
        slots_[s].steps_launched += n;
        ensure_growth(s, slots_[s].steps_launched + 1);
    }
    if (grid_grow_ == 0) {
        launch_step(); // sizes the grids; one cycle
        n--;
    }
    build_graph();
    cudaStream_t st = S(stream_);
    int full = n / graph_steps_, rest = n % graph_steps_;
    for (int q = 0; q < full; q++)
        CUDA_OK(cudaGraphLaunch((cudaGraphExec_t)graph_exec_, st));
    launches_ += (unsigned long long)full * (1 + 4ull * graph_steps_);
    launch_cycles(rest);
    CUDA_OK(cudaGetLastError());
}

void Pool::sync_state() {
    CUDA_OK(cudaSetDevice(device_));
    cudaStream_t st = S(stream_);
    if (!host_desc_.empty())
        CUDA_OK(cudaMemcpyAsync(host_desc_.data(), ddesc_, sizeof(DomainDesc) * host_desc_.size(),
                                cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
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
    if (grid_grow_ == 0) {
        launch_step();
        n--;
        cycles_launched_++;
    }
    for (int s = 0; s < (int)slots_.size(); s++) {
        if (!slots_[s].used)
            continue;
        slots_[s].steps_launched += n;
        ensure_growth(s, slots_[s].steps_launched + 1);
    }
    cudaStream_t st = S(stream_);
    cudaEvent_t ev[6];
    for (auto &e : ev)
        CUDA_OK(cudaEventCreate(&e));
    for (int q = 0; q < n; q++) {
        CUDA_OK(cudaEventRecord(ev[0], st));
        k_step_begin<<<1, kBlock, 0, st>>>(dstate_);
        CUDA_OK(cudaEventRecord(ev[1], st));
        k_grow<<<grid_grow_, kBlock, 0, st>>>(dstate_);
        CUDA_OK(cudaEventRecord(ev[2], st));
        k_claim<<<grid_claim_, kBlock, 0, st>>>(dstate_);
        CUDA_OK(cudaEventRecord(ev[3], st));
        k_capture<<<grid_capture_, kBlock, 0, st>>>(dstate_);
        CUDA_OK(cudaEventRecord(ev[4], st));
        k_neighbours<false><<<grid_nb_, kBlock, 0, st>>>(dstate_);
        CUDA_OK(cudaEventRecord(ev[5], st));
        CUDA_OK(cudaEventSynchronize(ev[5]));
        float t[5];
        for (int k = 0; k < 5; k++)
            CUDA_OK(cudaEventElapsedTime(&t[k], ev[k], ev[k + 1]));
        kt.begin_ms += t[0];
        kt.grow_ms += t[1];
        kt.claim_ms += t[2];
        kt.capture_ms += t[3];
        kt.neighbours_ms += t[4];
    }
    for (auto &e : ev)
        CUDA_OK(cudaEventDestroy(e));
    kt.cycles = n;
    cycles_launched_ += n;
    launches_ += 5ull * n;
    return kt;
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

void Pool::copy_out_raw(int slot, int32_t *grain_id, int8_t *cell_type) {
    CUDA_OK(cudaSetDevice(device_));
    const DomainDesc &d = host_desc_.at(slot);
    size_t N = slots_.at(slot).problem->g.domain_size;
    cudaStream_t st = S(stream_);
    if (grain_id)
        CUDA_OK(cudaMemcpyAsync(grain_id, d.gid, N * 4, cudaMemcpyDeviceToHost, st));
    if (cell_type)
        CUDA_OK(cudaMemcpyAsync(cell_type, d.ctype, N, cudaMemcpyDeviceToHost, st));
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
    size_t A = slots_.at(slot).problem->g.active_size;
    cudaStream_t st = S(stream_);
    if (dl)
        CUDA_OK(cudaMemcpyAsync(dl, d.dl, A * 4, cudaMemcpyDeviceToHost, st));
    if (doc)
        CUDA_OK(cudaMemcpyAsync(doc, d.doc, A * 12, cudaMemcpyDeviceToHost, st));
    if (cdl)
        CUDA_OK(cudaMemcpyAsync(cdl, d.cdl, A * 104, cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
}

void Pool::copy_out(int slot, int32_t *grain_id, int32_t *cell_type) {
    size_t N = slots_.at(slot).problem->g.domain_size;
    std::vector<int8_t> ct;
    if (cell_type)
        ct.resize(N);
    copy_out_raw(slot, grain_id, cell_type ? ct.data() : nullptr);
    if (cell_type)
        for (size_t i = 0; i < N; i++)
            cell_type[i] = ct[i];
}

int Pool::run_plain(int slot, std::string &log, double *nucl_s, double *capture_s) {
    // src/runCA.cpp:283-342 for one layer
    const Problem &p = *slots_.at(slot).problem;
    bool jump_type = p.cfg.simulation_type == "S" || p.cfg.simulation_type == "R";
    auto t0 = std::chrono::steady_clock::now();
    cudaEvent_t ev0, ev1;
    CUDA_OK(cudaEventCreate(&ev0));
    CUDA_OK(cudaEventCreate(&ev1));
    CUDA_OK(cudaEventRecord(ev0, S(stream_)));
    sync_state();
    int cycle = host_desc_[slot].cycle;
    while (true) {
        int n = 1000 - (cycle % 1000);
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
        if (c.superheated + c.undercooled == 0)
            break;
        if (jump_type && c.undercooled == 0) {
            unsigned long long next = c.next_cts;
            if ((next - (unsigned long long)(long long)cycle) > 5000) {
                int nc = (int)(next - 1);
                set_cycle(slot, nc);
                cycle = nc;
                log += "Jumping to cycle " + std::to_string(cycle + 1) + "\n";
            }
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

} // namespace exaca
