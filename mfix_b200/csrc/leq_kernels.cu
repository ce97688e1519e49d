// leq_kernels.cu -- sm_100a kernels of the LEQ_BICGS path (MFIX 2016-1,
// model/leq_bicgs.f and model/leqsol_mod.f), batch-shaped.
//
// Cell kernels walk a device table of TILE_CELLS-cell tiles.  Each tile's dot
// products are reduced inside the block and stored in a per-tile slot; the
// block that completes a system's last tile sums the slots in tile order and
// runs the scalar step of the iteration (alpha, omega, convergence test ...).
// The result is independent of which block finishes last and of what else is in
// the batch, so a system gives bit-identical results alone and in a mix.
//
// J-line kernels give each warp one or more whole lines (G lanes per line).
// Each lane eliminates a chunk of c consecutive rows to an interface form, the
// 2G interface rows are solved by parallel cyclic reduction over shuffles, and
// the interior rows are recovered in place.  Lines whose rows do not satisfy a
// local dominance bound (under which DGTSV never interchanges rows) are solved
// again by one lane with the exact pivoting DGTSV recurrence.
#include <cfloat>
#include <cstdio>
#include <algorithm>
#include <type_traits>

#include "leq_kernels.cuh"

#include <mutex>

namespace mfixgpu {

// ------------------------------------------------------------------ helpers
template <typename T>
__device__ __forceinline__ const T *diag_base(const SysDev &d);
template <>
__device__ __forceinline__ const double *diag_base<double>(const SysDev &d) { return d.a64; }
template <>
__device__ __forceinline__ const float *diag_base<float>(const SysDev &d) { return d.a32; }

template <typename T>
__device__ __forceinline__ T *vec(const SysDev &d, int id)
{
    return reinterpret_cast<T *>(d.vec[id]);
}

struct CellIdx {
    int i, j, k;  // 0-based
};

__device__ __forceinline__ CellIdx cell_ijk(const SysDev &d, uint32_t c)
{
    const uint32_t line = fdiv(c, d.div_j);
    CellIdx r;
    r.j = (int)(c - line * (uint32_t)d.jmax2);
    const uint32_t k = fdiv(line, d.div_i);
    r.k = (int)k;
    r.i = (int)(line - k * (uint32_t)d.imax2);
    return r;
}

// Layout of the arrays a kernel of element type T works on (SysDev::jp): the
// FP64 drop-in's are the caller's (pitch JMAX2, n cells), the mixed form's FP32
// arrays are padded (pitch jp, np cells).  j >= jmax2 marks a pad cell.
template <typename T>
__device__ __forceinline__ int pitch(const SysDev &d)
{
    return sizeof(T) == 4 ? d.jp : d.jmax2;
}
template <typename T>
__device__ __forceinline__ int64_t cells(const SysDev &d)
{
    return sizeof(T) == 4 ? d.np : d.n;
}
template <typename T>
__device__ __forceinline__ CellIdx cell_ijk_t(const SysDev &d, uint32_t c)
{
    if (sizeof(T) == 8) return cell_ijk(d, c);
    const uint32_t line = fdiv(c, d.div_jp);
    CellIdx r;
    r.j = (int)(c - line * (uint32_t)d.jp);
    const uint32_t k = fdiv(line, d.div_i);
    r.k = (int)k;
    r.i = (int)(line - k * (uint32_t)d.imax2);
    return r;
}

// Index in the mixed form's padded FP32 arrays of natural cell c.
__device__ __forceinline__ int64_t padded(const SysDev &d, int64_t c)
{
    const uint32_t line = fdiv((uint32_t)c, d.div_j);
    return c + (int64_t)line * (d.jp - d.jmax2);
}
// Natural cell of padded index p (-1 for a pad cell).
__device__ __forceinline__ int64_t natural(const SysDev &d, int64_t p)
{
    const uint32_t line = fdiv((uint32_t)p, d.div_jp);
    const int j = (int)(p - (int64_t)line * d.jp);
    return j < d.jmax2 ? (int64_t)line * d.jmax2 + j : -1;
}

// Neighbour increments of a serial box (model/set_increments.f:73-113), in cells
// of one axis: clamped at the array edge, or, along a cyclic axis, wrapping the
// interior cells 1..m-2 (0-based t, extent m with the wall layer): IP1(I) =
// IMAP_C(IMAP_C(I)+1) with IMAP_C(IMAX2) = IMIN1 and IMAP_C(IMIN2) = IMAX1
// (model/dmp_modules/gridmap_mod.f:496-503).
__device__ __forceinline__ int inc_m(int t, int m, bool cyc)
{
    if (cyc && t >= 1 && t <= m - 2) return t == 1 ? m - 3 : -1;
    return t > 0 ? -1 : 0;
}
__device__ __forceinline__ int inc_p(int t, int m, bool cyc)
{
    if (cyc && t >= 1 && t <= m - 2) return t == m - 2 ? -(m - 3) : 1;
    return t < m - 1 ? 1 : 0;
}

// 7-point product of row c with x, in the operand order of LEQ_MATVEC
// (model/leqsol_mod.f:240-250), neighbours clamped at the array edge.
template <typename T, typename TX>
__device__ __forceinline__ double stencil_row(const SysDev &d, const T *__restrict__ a, const TX *__restrict__ x,
                                              uint32_t c, const CellIdx &q)
{
    const int64_t n = d.n;
    const int64_t c1 = d.jmax2, c2 = (int64_t)d.jmax2 * d.imax2;
    const int64_t jm = inc_m(q.j, d.jmax2, d.cyc & 2), jp = inc_p(q.j, d.jmax2, d.cyc & 2);
    const int64_t im = inc_m(q.i, d.imax2, d.cyc & 1) * c1, ip = inc_p(q.i, d.imax2, d.cyc & 1) * c1;
    const int64_t p = c;
    using A = typename std::conditional<(sizeof(T) > sizeof(TX)), T, TX>::type;
    A v = (A)a[1 * n + p] * (A)x[p + jm];          // A(-2) * x(j-1)
    v = v + (A)a[2 * n + p] * (A)x[p + im];        // A(-1) * x(i-1)
    v = v + (A)a[3 * n + p] * (A)x[p];             // A( 0) * x
    v = v + (A)a[4 * n + p] * (A)x[p + ip];        // A( 1) * x(i+1)
    v = v + (A)a[5 * n + p] * (A)x[p + jp];        // A( 2) * x(j+1)
    if (d.do_k) {
        const int64_t km = inc_m(q.k, d.kmax2, d.cyc & 4) * c2, kp = inc_p(q.k, d.kmax2, d.cyc & 4) * c2;
        v = v + (A)a[0 * n + p] * (A)x[p + km];    // A(-3) * x(k-1)
        v = v + (A)a[6 * n + p] * (A)x[p + kp];    // A( 3) * x(k+1)
    }
    return (double)v;
}

template <int NV>
__device__ __forceinline__ void warp_sum(double (&v)[NV])
{
#pragma unroll
    for (int q = 0; q < NV; ++q)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
}

// The barrier of a reduction: the whole block (BAR = 0), or named barrier BAR
// over the first NT threads (kernels whose other warps do other work).
template <int BAR, int NT>
__device__ __forceinline__ void bsync()
{
    if constexpr (BAR == 0)
        __syncthreads();
    else
        asm volatile("bar.sync %0, %1;\n" ::"n"(BAR), "n"(NT) : "memory");
}

// Reduce v over the block (or the first NT threads, BAR > 0); thread 0 receives
// the total in v.
template <int NV, int BAR = 0, int NT = 0>
__device__ __forceinline__ void block_sum(double (&v)[NV])
{
    __shared__ double red[NV][32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = BAR ? NT >> 5 : blockDim.x >> 5;
    warp_sum<NV>(v);
    bsync<BAR, NT>();
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NV; ++q) red[q][warp] = v[q];
    bsync<BAR, NT>();
    if (warp == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) v[q] = lane < nw ? red[q][lane] : 0.0;
        warp_sum<NV>(v);
    }
}

// Deterministic per-system reductions.  Each tile's sum is formed in a fixed
// order and stored in the tile's slot; once every tile of a system has
// arrived, the block that completed it adds the slots in tile order.  Arrivals
// are counted once per run of consecutive tiles of one system a block has
// processed (one fence and one atomic per run instead of per tile).
struct TileRun {
    int sys;
    int count;
};

template <int NV, int BAR = 0, int NT = 0>
__device__ __forceinline__ void tile_partial(const BatchView &b, const SysDev &d, int tile_idx, double (&v)[NV])
{
    block_sum<NV, BAR, NT>(v);
    if (threadIdx.x == 0) {
        double *slot = b.partials + 2 * (int64_t)(d.tile_base + tile_idx);
#pragma unroll
        for (int q = 0; q < NV; ++q) slot[q] = v[q];
    }
}

// Reports the run's tiles; the block that completes the system's count forms
// the totals and calls fin(state, totals) on thread 0.
template <int NV, int BAR = 0, int NT = 0, typename Fin>
__device__ __forceinline__ void run_close(const BatchView &b, TileRun &run, Fin &fin)
{
    if (run.count == 0) return;
    __shared__ int last;
    const SysDev &d = b.sys[run.sys];
    SysState &st = b.st[run.sys];
    if (threadIdx.x == 0) {
        __threadfence();  // this thread's slot stores before the arrival count
        const unsigned prev = atomicAdd(&st.arrivals, (unsigned)run.count);
        last = (prev + (unsigned)run.count == (unsigned)d.ntiles);
    }
    bsync<BAR, NT>();
    run.count = 0;
    if (!last) return;
    __threadfence();
    double acc[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) acc[q] = 0.0;
    for (int t = threadIdx.x; t < d.ntiles; t += (BAR ? NT : (int)blockDim.x)) {
        const double *slot = b.partials + 2 * (int64_t)(d.tile_base + t);
#pragma unroll
        for (int q = 0; q < NV; ++q) acc[q] += __ldcg(slot + q);
    }
    block_sum<NV, BAR, NT>(acc);
    if (threadIdx.x == 0) {
        st.arrivals = 0;
        fin(st, acc);
    }
}

template <int NV, int BAR = 0, int NT = 0, typename Fin>
__device__ __forceinline__ void run_add(const BatchView &b, TileRun &run, int sys, Fin &fin)
{
    if (run.sys != sys) {
        run_close<NV, BAR, NT>(b, run, fin);
        run.sys = sys;
    }
    run.count += 1;
}

// ------------------------------------------------------------------ scalar steps
// model/leq_bicgs.f:485-495 (the REAL() casts are single-precision conversions).
__device__ inline void final_logic(SysState &s, bool converged)
{
    if (!converged) converged = ((double)(float)s.rnorm <= s.tol * s.rnorm0);
    s.ier = 0;
    s.exit_kind = converged ? EX_RNORM : EX_ITMAX;
    if (!converged) {
        s.ier = -1;
        s.iter_tot_add = s.iter;
        if ((double)(float)s.rnorm >= (double)0.2f * (double)(float)s.rnorm0) s.ier = -2;
    }
    s.status = ST_DONE;
}

// End of the setup: Rnorm0 (model/leq_bicgs.f:291).
__device__ inline void fin_rnorm0(SysState &s, double rr) { s.rnorm0 = sqrt(rr); }

// Entry to the main loop: rho(0) and its zero test (:315-332).
__device__ inline void fin_rho0(SysState &s, double rtr)
{
    s.i = 1;
    s.iter = 1;
    s.rnorm = 0.0;
    s.snorm_exit = 0;
    s.phase = PH_INNER;
    if (s.itmax < 1) {
        final_logic(s, false);
        return;
    }
    s.rho = rtr;
    if (rtr == 0.0) {
        s.ier = 0;
        s.exit_kind = EX_RHO0;
        s.status = ST_DONE;
    }
}

// ------------------------------------------------------------------ setup kernels
// Unit-diagonal scaling of every row (model/leq_bicgs.f:211-226).
__global__ void k_scale(BatchView b)
{
    for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
        const Tile tl = b.tiles[t];
        const SysDev &d = b.sys[tl.sys];
        if (!gate_ok(b.st[tl.sys], G_SETUP)) continue;
        const int64_t n = d.n;
        const int64_t c0 = (int64_t)tl.idx * TILE_CELLS, c1 = min(n, c0 + TILE_CELLS);
        int bad = 0;
        #pragma unroll 4
        for (int64_t c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
            double m = fabs(d.a64[c]);
#pragma unroll
            for (int q = 1; q < 7; ++q) {
                const double v = fabs(d.a64[q * n + c]);
                if (isnan(m) || v > m) m = v;
            }
            if (m > 0.0) {
                const double oam = 1.0 / m;
#pragma unroll
                for (int q = 0; q < 7; ++q) d.a64[q * n + c] = d.a64[q * n + c] * oam;
                d.b64[c] = d.b64[c] * oam;
            } else {
                bad = 1;
            }
        }
        if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(&b.st[tl.sys].err, 1);
    }
}

// A singular row returns IER = -2 before any iteration (:232-233).
__global__ void k_after_scale(BatchView b)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= b.nsys) return;
    SysState &st = b.st[s];
    if (!gate_ok(st, G_SETUP)) return;
    if (st.err & 1) {
        st.ier = -2;
        st.exit_kind = EX_SINGULAR;
        st.status = ST_DONE;
        return;
    }
    st.phase = PH_INIT;
}

// LEQ_CG0 (model/leq_cg.f): IER rules after the loop (:443-450): REAL() values in the ratio test.
__device__ inline void cg_final(SysState &s)
{
    s.ier = -1;
    s.iter_tot_add = s.iter;
    if ((double)(float)s.rnorm >= (double)0.2f * (double)(float)s.rnorm0) s.ier = -2;
    s.exit_kind = EX_ITMAX;
    s.status = ST_DONE;
}

// Entry to the loop (:269-271).
__device__ inline void cg_begin(SysState &s)
{
    s.i = 1;
    s.iter = 1;
    s.rnorm = 0.0;
    s.phase = PH_INNER;
    if (s.itmax < 1) cg_final(s);
}

// End of the setup: the FP64 drop-in enters the loop (its Rtilde step already
// moved it to PH_INNER unless it finished), the mixed form starts with an FP64 update.
__global__ void k_init_done(BatchView b)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= b.nsys) return;
    SysState &st = b.st[s];
    if (!gate_ok(st, G_INIT)) return;
    if (st.method == 5) {  // LEQ_CG0
        cg_begin(st);
        return;
    }
    if (st.method == 3) {  // LEQ_GMRES0: the host drives the iteration; the sweeps run in PH_INNER
        st.phase = PH_INNER;
        return;
    }
    // a nearly singular operator (pressure correction) is deflated (k_defl_setup);
    // where that is off or impossible it goes to the FP64 drop-in before any FP32
    // iteration: its undeflated FP32 Krylov process stagnates
    if (st.mixed && __uint_as_float(st.margin_bits) < st.min_margin && !st.defl) {
        st.exit_kind = EX_FALLBACK;
        st.ier = -20;
        st.status = ST_DONE;
        return;
    }
    st.phase = st.mixed ? PH_OUTER : PH_INNER;
}

// Mixed form's FP32 operator: the scaled diagonals rounded to FP32, and each
// row's sum formed in FP64 first.  The FP32 matvec evaluates
//   sum_nb a_nb (x_nb - x) + defect * x,
// algebraically the same as the seven products, but exact to FP32 rounding in
// the smooth (near-null) mode of nearly singular operators such as pressure
// correction, where the seven products cancel to a millionth of their size.
__global__ void k_to_f32(BatchView b)
{
    for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
        const Tile tl = b.tiles[t];
        const SysDev &d = b.sys[tl.sys];
        if (!gate_ok(b.st[tl.sys], G_INIT)) continue;
        const int64_t n = d.n, np = d.np;
        const int64_t p0 = (int64_t)tl.idx * TILE_CELLS, p1 = min(np, p0 + TILE_CELLS);
        float margin = __int_as_float(0x7f800000);  // +inf
        #pragma unroll 4
        for (int64_t p = p0 + threadIdx.x; p < p1; p += blockDim.x) {
            const int64_t c = natural(d, p);
            if (c < 0) {  // pad cell of the padded FP32 arrays: zeros, A(0) = 1
#pragma unroll
                for (int q = 0; q < 7; ++q) d.a32[q * np + p] = q == 3 ? 1.f : 0.f;
                d.defect[p] = 0.f;
                d.defl_z[p] = 0;
                d.defl_az[p] = 0.f;
#pragma unroll
                for (int v = V_R; v < NVEC; ++v) reinterpret_cast<float *>(d.vec[v])[p] = 0.f;
                continue;
            }
            double sum = 0.0;
            bool coupled = false;
#pragma unroll
            for (int q = 0; q < 7; ++q) {
                const double v = d.a64[q * n + c];
                d.a32[q * np + p] = (float)v;
                if (d.do_k || (q != 0 && q != 6)) {
                    sum += v;
                    if (q != 3 && v != 0.0) coupled = true;
                }
            }
            d.defect[p] = (float)sum;  // the row sum, exact to FP32 rounding however small
            d.defl_z[p] = coupled ? 1 : 0;
            const double a0 = fabs(d.a64[3 * n + c]);
            if (a0 > 0.0) margin = fminf(margin, (float)(fabs(sum) / a0));
        }
        // the system's smallest margin (order-free, so the same in any batch)
        for (int o = 16; o > 0; o >>= 1) margin = fminf(margin, __shfl_xor_sync(0xffffffffu, margin, o));
        if ((threadIdx.x & 31) == 0) atomicMin(&b.st[tl.sys].margin_bits, __float_as_uint(margin));
    }
}

// Deflation of the near-null mode (mixed form, systems whose diagonal-dominance
// margin is below min_margin: pressure correction, where the rows of coupled
// cells sum to a millionth of their diagonal).  z is 1 on the rows coupled to a
// neighbour and 0 on decoupled (wall) rows; the preconditioner becomes
//   Phat = M^{-1} P + c z,  c = z^T P / z^T A z,
// so that the constant mode over the coupled cells, which the line sweeps barely
// reduce, is solved exactly in every application.  This kernel forms A z in FP64
// (stored in FP32) and E = z^T A z.
__global__ void k_defl_setup(BatchView b)
{
    TileRun run{-1, 0};
    auto fin = [&](SysState &st, const double(&tot)[1]) {
        st.defl_e = tot[0];
        st.defl = (tot[0] != 0.0 && isfinite(tot[0])) ? 1 : 0;
    };
    for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
        const Tile tl = b.tiles[t];
        const SysDev &d = b.sys[tl.sys];
        SysState &st = b.st[tl.sys];
        if (!gate_ok(st, G_INIT) || !st.mixed || !st.defl_allow ||
            !(__uint_as_float(st.margin_bits) < st.min_margin))
            continue;
        const int64_t p0 = (int64_t)tl.idx * TILE_CELLS, p1 = min(d.np, p0 + TILE_CELLS);
        const int64_t n = d.n, c1 = d.jp, c2 = (int64_t)d.jp * d.imax2;
        double v[1] = {0.0};
        #pragma unroll 2
        for (int64_t p = p0 + threadIdx.x; p < p1; p += blockDim.x) {
            const int64_t c = natural(d, p);
            if (c < 0) continue;  // pad cell (A z = 0 there)
            // A z in the operand order of LEQ_MATVEC: FP64 diagonals at the natural
            // cell, z at the padded neighbours (clamped at the array edge)
            const CellIdx q = cell_ijk_t<float>(d, (uint32_t)p);
            const unsigned char *z = d.defl_z;
            const int64_t jm = inc_m(q.j, d.jmax2, d.cyc & 2), jq = inc_p(q.j, d.jmax2, d.cyc & 2);
            const int64_t im = inc_m(q.i, d.imax2, d.cyc & 1) * c1, ip = inc_p(q.i, d.imax2, d.cyc & 1) * c1;
            double az = d.a64[1 * n + c] * (double)z[p + jm];
            az = az + d.a64[2 * n + c] * (double)z[p + im];
            az = az + d.a64[3 * n + c] * (double)z[p];
            az = az + d.a64[4 * n + c] * (double)z[p + ip];
            az = az + d.a64[5 * n + c] * (double)z[p + jq];
            if (d.do_k) {
                const int64_t km = inc_m(q.k, d.kmax2, d.cyc & 4) * c2, kp = inc_p(q.k, d.kmax2, d.cyc & 4) * c2;
                az = az + d.a64[0 * n + c] * (double)z[p + km];
                az = az + d.a64[6 * n + c] * (double)z[p + kp];
            }
            d.defl_az[p] = (float)az;
            if (z[p]) v[0] += az;
        }
        tile_partial<1>(b, d, tl.idx, v);
        run_add<1>(b, run, tl.sys, fin);
    }
    run_close<1>(b, run, fin);
}

// R = B - A*Var and ||R|| (model/leq_bicgs.f:283-291).
template <typename T>
__global__ void k_init_residual(BatchView b)
{
    TileRun run{-1, 0};
    auto fin = [&](SysState &st, const double(&tot)[1]) { fin_rnorm0(st, tot[0]); };
    for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
        const Tile tl = b.tiles[t];
        const SysDev &d = b.sys[tl.sys];
        SysState &st = b.st[tl.sys];
        if (!gate_ok(st, G_INIT)) continue;
        const int64_t c0 = (int64_t)tl.idx * TILE_CELLS, c1 = min(d.n, c0 + TILE_CELLS);
        const T *a = diag_base<T>(d);
        const T *x = vec<T>(d, V_X);
        T *r = vec<T>(d, V_R);
        double v[1] = {0.0};
        #pragma unroll 4
        for (int64_t c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
            const CellIdx q = cell_ijk(d, (uint32_t)c);
            const T ax = (T)stencil_row<T, T>(d, a, x, (uint32_t)c, q);
            const T rv = (T)d.b64[c] - ax;
            r[c] = rv;
            v[0] += (double)rv * (double)rv;
        }
        tile_partial<1>(b, d, tl.idx, v);
        run_add<1>(b, run, tl.sys, fin);
    }
    run_close<1>(b, run, fin);
}

__device__ __forceinline__ uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// The counter-based stream that replaces RANDOM_NUMBER (model/leq_bicgs.f:298).
__device__ __forceinline__ double uniform01(uint64_t seed, uint64_t tag, uint64_t idx)
{
    const uint64_t key = mix64(seed * 0x9E3779B97F4A7C15ULL + tag * 0xD1B54A32D192ED03ULL + 0x632BE59BD9B4E019ULL);
    const uint64_t v = mix64(key + (idx + 1) * 0x9E3779B97F4A7C15ULL);
    return (double)(v >> 11) * 0x1.0p-53;
}

// Rtilde = R + (2u-1)*1e-6*Rnorm0 (:303-305) and rho(0) = (Rtilde, R) (:318).
template <typename T>
__global__ void k_init_rtilde(BatchView b, uint64_t seed)
{
    TileRun run{-1, 0};
    auto fin = [&](SysState &st, const double(&tot)[1]) { fin_rho0(st, tot[0]); };
    for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
        const Tile tl = b.tiles[t];
        const SysDev &d = b.sys[tl.sys];
        SysState &st = b.st[tl.sys];
        if (!gate_ok(st, G_INIT)) continue;
        const int64_t c0 = (int64_t)tl.idx * TILE_CELLS, c1 = min(d.n, c0 + TILE_CELLS);
        const double rn0 = st.rnorm0;
        const T *r = vec<T>(d, V_R);
        T *rt = vec<T>(d, V_RT);
        double v[1] = {0.0};
        #pragma unroll 4
        for (int64_t c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
            const double u = uniform01(seed, 0xA1, (uint64_t)c);
            const T rv = r[c];
            const T rtv = (T)((double)rv + (2.0 * u - 1.0) * 1.0e-6 * rn0);
            rt[c] = rtv;
            v[0] += (double)rtv * (double)rv;
        }
        tile_partial<1>(b, d, tl.idx, v);
        run_add<1>(b, run, tl.sys, fin);
    }
    run_close<1>(b, run, fin);
}

// ------------------------------------------------------------------ iteration kernels
// Every cell kernel is persistent (grid = resident blocks) and strides over the
// batch's tiles.  Inside a tile each thread first loads the operands of U cells
// into registers and only then computes and stores, so the loads of U cells are
// in flight together (the stores could otherwise alias the next cells' loads and
// serialize them).

// Clamped neighbour offsets of cell c (model/set_increments.f:80-109).
struct Offs {
    int64_t jm, jp, im, ip, km, kp;
};

template <typename T = double>
__device__ __forceinline__ Offs cell_offs(const SysDev &d, uint32_t c, int *jout = nullptr)
{
    const CellIdx q = cell_ijk_t<T>(d, c);
    if (jout) *jout = q.j;
    const int64_t c1 = pitch<T>(d), c2 = (int64_t)pitch<T>(d) * d.imax2;
    Offs o;
    o.jm = inc_m(q.j, d.jmax2, d.cyc & 2);
    o.jp = inc_p(q.j, d.jmax2, d.cyc & 2);
    o.im = inc_m(q.i, d.imax2, d.cyc & 1) * c1;
    o.ip = inc_p(q.i, d.imax2, d.cyc & 1) * c1;
    o.km = d.do_k ? inc_m(q.k, d.kmax2, d.cyc & 4) * c2 : 0;
    o.kp = d.do_k ? inc_p(q.k, d.kmax2, d.cyc & 4) * c2 : 0;
    return o;
}

// The seven operands of row c of A*x: a[0..6] = A(-2), A(-1), A(0), A(1), A(2), A(-3), A(3)
// (the order LEQ_MATVEC adds them in, model/leqsol_mod.f:240-250), x alike.
template <typename T>
struct Row7 {
    T a[7], x[7];
};

// T = float: the mixed form's padded FP32 arrays; *jout receives the row's j
// (j >= JMAX2 marks a pad cell, whose product the caller discards).
template <typename T, typename TX, bool DEFECT = false>
__device__ __forceinline__ void load_row7(const SysDev &d, const T *__restrict__ A, const TX *__restrict__ X,
                                          int64_t c, Row7<T> &r, int *jout = nullptr)
{
    const int64_t n = cells<T>(d);
    const Offs o = cell_offs<T>(d, (uint32_t)c, jout);
    r.a[0] = A[1 * n + c];
    r.x[0] = (T)X[c + o.jm];
    r.a[1] = A[2 * n + c];
    r.x[1] = (T)X[c + o.im];
    if constexpr (DEFECT)
        r.a[2] = (T)d.defect[c];
    else
        r.a[2] = A[3 * n + c];
    r.x[2] = (T)X[c];
    r.a[3] = A[4 * n + c];
    r.x[3] = (T)X[c + o.ip];
    r.a[4] = A[5 * n + c];
    r.x[4] = (T)X[c + o.jp];
    if (d.do_k) {
        r.a[5] = A[0 * n + c];
        r.x[5] = (T)X[c + o.km];
        r.a[6] = A[6 * n + c];
        r.x[6] = (T)X[c + o.kp];
    } else {
        r.a[5] = r.a[6] = T(0);
        r.x[5] = r.x[6] = T(0);
    }
}

// The defect form's terms with every rounding stated (a fused multiply-add per
// term), so that each kernel forming the product gets the same bits whatever
// the compiler would contract.
__device__ __forceinline__ float dterm0(float a, float xn, float xc) { return __fmul_rn(a, __fsub_rn(xn, xc)); }
__device__ __forceinline__ float dterm(float acc, float a, float xn, float xc)
{
    return __fmaf_rn(a, __fsub_rn(xn, xc), acc);
}
__device__ __forceinline__ float dcentre(float acc, float rowsum, float xc) { return __fmaf_rn(rowsum, xc, acc); }

template <typename T, bool DEFECT = false>
__device__ __forceinline__ T dot_row7(const Row7<T> &r, bool do_k)
{
    if constexpr (DEFECT) {  // a[2] holds the row sum (mixed form: T = float)
        const T xc = r.x[2];
        T v = dterm0(r.a[0], r.x[0], xc);
        v = dterm(v, r.a[1], r.x[1], xc);
        v = dcentre(v, r.a[2], xc);
        v = dterm(v, r.a[3], r.x[3], xc);
        v = dterm(v, r.a[4], r.x[4], xc);
        if (do_k) {
            v = dterm(v, r.a[5], r.x[5], xc);
            v = dterm(v, r.a[6], r.x[6], xc);
        }
        return v;
    }
    T v = r.a[0] * r.x[0];
    v = v + r.a[1] * r.x[1];
    v = v + r.a[2] * r.x[2];
    v = v + r.a[3] * r.x[3];
    v = v + r.a[4] * r.x[4];
    if (do_k) {
        v = v + r.a[5] * r.x[5];
        v = v + r.a[6] * r.x[6];
    }
    return v;
}

// Two neighbouring cells per thread: 8-byte (FP32) or 16-byte (FP64) loads
// halve the load instructions a streaming kernel needs for the same bytes.
// Tiles start at multiples of TILE_CELLS and vectors at 256-byte boundaries,
// so the pair (c, c+1) with c even is aligned.
template <typename T>
struct Vec2;
template <>
struct Vec2<float> {
    using type = float2;
};
template <>
struct Vec2<double> {
    using type = double2;
};
template <typename T>
using vec2_t = typename Vec2<T>::type;

template <typename T>
__device__ __forceinline__ vec2_t<T> ld2(const T *p)
{
    return *reinterpret_cast<const vec2_t<T> *>(p);
}
template <typename T>
__device__ __forceinline__ void st2(T *p, const vec2_t<T> &v)
{
    *reinterpret_cast<vec2_t<T> *>(p) = v;
}
template <typename T>
__device__ __forceinline__ vec2_t<T> mk2(T a, T b)
{
    vec2_t<T> r;
    r.x = a;
    r.y = b;
    return r;
}

// The operands of rows c and c+1 (c even) of one J-line.  Used when JMAX2 is
// even: then both cells share i and k, DIMENSION_3 is even so every diagonal's
// pair is aligned, and so are the pairs at the i and k neighbours.  (A pair
// form for odd JMAX2, whose cells may straddle two lines, needs one-by-one loads
// of the i and k neighbours; in the same kernel it slowed the even form by
// 10-25%.)
template <typename T>
__device__ __forceinline__ bool pair_rows(const SysDev &d) { return (pitch<T>(d) & 1) == 0; }

template <typename T>
struct Pair7 {
    vec2_t<T> a[7], x[7];
};

template <typename T, bool DEFECT = false>
__device__ __forceinline__ void load_pair7(const SysDev &d, const T *__restrict__ A, const T *__restrict__ X,
                                           int64_t c, Pair7<T> &r, int *jout = nullptr)
{
    const int64_t n = cells<T>(d);
    const CellIdx q = cell_ijk_t<T>(d, (uint32_t)c);
    if (jout) *jout = q.j;
    const int64_t c1 = pitch<T>(d), c2 = (int64_t)pitch<T>(d) * d.imax2;
    const int64_t im = inc_m(q.i, d.imax2, d.cyc & 1) * c1, ip = inc_p(q.i, d.imax2, d.cyc & 1) * c1;
    const vec2_t<T> xc = ld2(X + c);
    // x(j-1) of cell c and x(j+1) of cell c+1 (the pair's own cells otherwise);
    // along a cyclic J both cells' J neighbours may wrap
    const bool cj = (d.cyc & 2) != 0;
    const T xl = X[c + inc_m(q.j, d.jmax2, cj)];
    const T xr = X[c + 1 + inc_p(q.j + 1, d.jmax2, cj)];
    r.a[0] = ld2(A + 1 * n + c);
    r.x[0] = mk2<T>(xl, cj ? X[c + 1 + inc_m(q.j + 1, d.jmax2, true)] : xc.x);
    r.a[1] = ld2(A + 2 * n + c);
    r.x[1] = ld2(X + c + im);
    if constexpr (DEFECT)
        r.a[2] = ld2(reinterpret_cast<const T *>(d.defect) + c);
    else
        r.a[2] = ld2(A + 3 * n + c);
    r.x[2] = xc;
    r.a[3] = ld2(A + 4 * n + c);
    r.x[3] = ld2(X + c + ip);
    r.a[4] = ld2(A + 5 * n + c);
    r.x[4] = mk2<T>(cj ? X[c + inc_p(q.j, d.jmax2, true)] : xc.y, xr);
    if (d.do_k) {
        const int64_t km = inc_m(q.k, d.kmax2, d.cyc & 4) * c2, kp = inc_p(q.k, d.kmax2, d.cyc & 4) * c2;
        r.a[5] = ld2(A + 0 * n + c);
        r.x[5] = ld2(X + c + km);
        r.a[6] = ld2(A + 6 * n + c);
        r.x[6] = ld2(X + c + kp);
    } else {
        r.a[5] = r.a[6] = mk2<T>(T(0), T(0));
        r.x[5] = r.x[6] = mk2<T>(T(0), T(0));
    }
}

// dot_row7 of both rows, in the same operand order
template <typename T, bool DEFECT = false>
__device__ __forceinline__ vec2_t<T> dot_pair7(const Pair7<T> &r, bool do_k)
{
    if constexpr (DEFECT) {  // a[2] holds the row sums (mixed form: T = float)
        const T cx = r.x[2].x, cy = r.x[2].y;
        T u = dterm0(r.a[0].x, r.x[0].x, cx);
        T w = dterm0(r.a[0].y, r.x[0].y, cy);
        u = dterm(u, r.a[1].x, r.x[1].x, cx);
        w = dterm(w, r.a[1].y, r.x[1].y, cy);
        u = dcentre(u, r.a[2].x, cx);
        w = dcentre(w, r.a[2].y, cy);
        u = dterm(u, r.a[3].x, r.x[3].x, cx);
        w = dterm(w, r.a[3].y, r.x[3].y, cy);
        u = dterm(u, r.a[4].x, r.x[4].x, cx);
        w = dterm(w, r.a[4].y, r.x[4].y, cy);
        if (do_k) {
            u = dterm(u, r.a[5].x, r.x[5].x, cx);
            w = dterm(w, r.a[5].y, r.x[5].y, cy);
            u = dterm(u, r.a[6].x, r.x[6].x, cx);
            w = dterm(w, r.a[6].y, r.x[6].y, cy);
        }
        return mk2<T>(u, w);
    }
    T u = r.a[0].x * r.x[0].x;
    T w = r.a[0].y * r.x[0].y;
    u = u + r.a[1].x * r.x[1].x;
    w = w + r.a[1].y * r.x[1].y;
    u = u + r.a[2].x * r.x[2].x;
    w = w + r.a[2].y * r.x[2].y;
    u = u + r.a[3].x * r.x[3].x;
    w = w + r.a[3].y * r.x[3].y;
    u = u + r.a[4].x * r.x[4].x;
    w = w + r.a[4].y * r.x[4].y;
    if (do_k) {
        u = u + r.a[5].x * r.x[5].x;
        w = w + r.a[5].y * r.x[5].y;
        u = u + r.a[6].x * r.x[6].x;
        w = w + r.a[6].y * r.x[6].y;
    }
    return mk2<T>(u, w);
}

// cells handled per thread per batch: streaming kernels
template <typename T>
struct Batch {
    static constexpr int STREAM = sizeof(T) == 8 ? 4 : 8;
};

// z^T v over a cell pair (deflated mixed systems)
template <typename T>
__device__ __forceinline__ double zdot2(const unsigned char *z, int64_t c, const vec2_t<T> &v)
{
    const uchar2 zz = *reinterpret_cast<const uchar2 *>(z + c);
    return (zz.x ? (double)v.x : 0.0) + (zz.y ? (double)v.y : 0.0);
}

// P = R (i = 1) or P = R + beta*(P - omega*V) (model/leq_bicgs.f:334-343).
// Deflated mixed systems also form c_p = z^T P / z^T A z.
template <typename T, bool MIXED>
__global__ void __launch_bounds__(256, 4) k_p_update(BatchView b)
{
    constexpr int U2 = Batch<T>::STREAM / 2;
    TileRun run{-1, 0};
    auto fin = [&](SysState &st, const double(&tot)[1]) { st.defl_cp = tot[0] / st.defl_e; };
    for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
        const Tile tl = b.tiles[t];
        const SysDev &d = b.sys[tl.sys];
        const SysState &st = b.st[tl.sys];
        if (!gate_ok(st, G_INNER)) continue;
        const int64_t c0 = (int64_t)tl.idx * TILE_CELLS;
        const int cnt = (int)min((int64_t)TILE_CELLS, cells<T>(d) - c0);
        const T *__restrict__ r = vec<T>(d, V_R) + c0;
        T *__restrict__ p = vec<T>(d, V_P) + c0;
        const int np = cnt >> 1;  // cell pairs; an odd last cell is done by thread 0
        const bool defl = MIXED && st.defl;
        double zv[1] = {0.0};
        if (st.i == 1) {
            for (int base = threadIdx.x; base < np; base += U2 * blockDim.x) {
                vec2_t<T> rv[U2];
#pragma unroll
                for (int u = 0; u < U2; ++u) {
                    const int q = base + u * blockDim.x;
                    if (q < np) rv[u] = ld2(r + 2 * q);
                }
#pragma unroll
                for (int u = 0; u < U2; ++u) {
                    const int q = base + u * blockDim.x;
                    if (q < np) {
                        st2(p + 2 * q, rv[u]);
                        if (defl) zv[0] += zdot2<T>(d.defl_z, c0 + 2 * q, rv[u]);
                    }
                }
            }
            if ((cnt & 1) && threadIdx.x == 0) {
                p[cnt - 1] = r[cnt - 1];
                if (defl && d.defl_z[c0 + cnt - 1]) zv[0] += (double)r[cnt - 1];
            }
        } else {
            const T beta = (T)st.beta, omega = (T)st.omega;
            const T *__restrict__ v = vec<T>(d, V_V) + c0;
            for (int base = threadIdx.x; base < np; base += U2 * blockDim.x) {
                vec2_t<T> rv[U2], pv[U2], vv[U2];
#pragma unroll
                for (int u = 0; u < U2; ++u) {
                    const int q = base + u * blockDim.x;
                    if (q < np) {
                        rv[u] = ld2(r + 2 * q);
                        pv[u] = ld2(p + 2 * q);
                        vv[u] = ld2(v + 2 * q);
                    }
                }
#pragma unroll
                for (int u = 0; u < U2; ++u) {
                    const int q = base + u * blockDim.x;
                    if (q < np) {
                        const vec2_t<T> pn = mk2<T>(rv[u].x + beta * (pv[u].x - omega * vv[u].x),
                                                    rv[u].y + beta * (pv[u].y - omega * vv[u].y));
                        st2(p + 2 * q, pn);
                        if (defl) zv[0] += zdot2<T>(d.defl_z, c0 + 2 * q, pn);
                    }
                }
            }
            if ((cnt & 1) && threadIdx.x == 0) {
                const int c = cnt - 1;
                p[c] = r[c] + beta * (p[c] - omega * v[c]);
                if (defl && d.defl_z[c0 + c]) zv[0] += (double)p[c];
            }
        }
        if (defl) {
            tile_partial<1>(b, d, tl.idx, zv);
            run_add<1>(b, run, tl.sys, fin);
        }
    }
    run_close<1>(b, run, fin);
}

// DIAG preconditioner, LEQ_MSOLVE1 (model/leqsol_mod.f:719-746): var = b / A(0).
template <typename T>
__global__ void __launch_bounds__(256, 4) k_diag(BatchView b, int src, int dst, int gate)
{
    constexpr int U = Batch<T>::STREAM;
    for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
        const Tile tl = b.tiles[t];
        const SysDev &d = b.sys[tl.sys];
        if (!gate_ok(b.st[tl.sys], gate)) continue;
        const int64_t c0 = (int64_t)tl.idx * TILE_CELLS;
        const int cnt = (int)min((int64_t)TILE_CELLS, cells<T>(d) - c0);
        const T *__restrict__ a0 = diag_base<T>(d) + 3 * cells<T>(d) + c0;
        const T *__restrict__ x = vec<T>(d, src) + c0;
        T *__restrict__ y = vec<T>(d, dst) + c0;
        for (int base = threadIdx.x; base < cnt; base += U * blockDim.x) {
            T xv[U], av[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int c = base + u * blockDim.x;
                if (c < cnt) {
                    xv[u] = x[c];
                    av[u] = a0[c];
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int c = base + u * blockDim.x;
                if (c < cnt) y[c] = xv[u] / av[u];
            }
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(256, 4) k_copy(BatchView b, int src, int dst, int gate)
{
    constexpr int U = Batch<T>::STREAM;
    for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
        const Tile tl = b.tiles[t];
        const SysDev &d = b.sys[tl.sys];
        if (!gate_ok(b.st[tl.sys], gate)) continue;
        const int64_t c0 = (int64_t)tl.idx * TILE_CELLS;
        const int cnt = (int)min((int64_t)TILE_CELLS, cells<T>(d) - c0);
        const T *__restrict__ x = vec<T>(d, src) + c0;
        T *__restrict__ y = vec<T>(d, dst) + c0;
        for (int base = threadIdx.x; base < cnt; base += U * blockDim.x) {
            T xv[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int c = base + u * blockDim.x;
                if (c < cnt) xv[u] = x[c];
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int c = base + u * blockDim.x;
                if (c < cnt) y[c] = xv[u];
            }
        }
    }
}

// V = A*Phat and alpha = rho / (Rtilde, V) (model/leq_bicgs.f:355-361).
template <typename T, bool MIXED, bool PAIR>
__global__ void __launch_bounds__(256) k_matvec_alpha(BatchView b, int src)
{
    constexpr int U = 2;  // one-cell rows: two cells per thread and pass (80 registers in FP32)
    constexpr int UP = 1;  // one cell pair per thread and pass: fewer registers, more resident warps
    TileRun run{-1, 0};
    auto fin = [&](SysState &st, const double(&tot)[1]) { st.alpha = st.rho / tot[0]; };
    for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
        const Tile tl = b.tiles[t];
        const SysDev &d = b.sys[tl.sys];
        SysState &st = b.st[tl.sys];
        if (!gate_ok(st, G_INNER) || pair_rows<T>(d) != PAIR) continue;
        const int64_t c0 = (int64_t)tl.idx * TILE_CELLS;
        const int cnt = (int)min((int64_t)TILE_CELLS, cells<T>(d) - c0);
        const T *__restrict__ a = diag_base<T>(d);
        const T *__restrict__ x = vec<T>(d, src);
        const T *__restrict__ rt = vec<T>(d, V_RT);
        T *__restrict__ y = vec<T>(d, V_V);
        double v[1] = {0.0};
        // deflated mixed systems: V = A (Phat + c_p z) = A Phat + c_p A z
        const bool defl = MIXED && st.defl;
        const double cp = defl ? st.defl_cp : 0.0;
        if constexpr (PAIR) {
            const int np = cnt >> 1;
            for (int base = threadIdx.x; base < np; base += UP * blockDim.x) {
                Pair7<T> rw[UP];
                int jr[UP];
                vec2_t<T> rtv[UP];
#pragma unroll
                for (int u = 0; u < UP; ++u) {
                    const int q = base + u * blockDim.x;
                    if (q < np) {
                        load_pair7<T, MIXED>(d, a, x, c0 + 2 * q, rw[u], &jr[u]);
                        rtv[u] = ld2(rt + c0 + 2 * q);
                    }
                }
#pragma unroll
                for (int u = 0; u < UP; ++u) {
                    const int q = base + u * blockDim.x;
                    if (q < np) {
                        vec2_t<T> yv = dot_pair7<T, MIXED>(rw[u], d.do_k);
                        if (jr[u] >= d.jmax2) yv.x = T(0);  // pad cells of the padded FP32 arrays
                        if (jr[u] + 1 >= d.jmax2) yv.y = T(0);
                        if (defl) {
                            const float2 az = ld2(d.defl_az + c0 + 2 * q);
                            yv.x = yv.x + (T)(cp * (double)az.x);
                            yv.y = yv.y + (T)(cp * (double)az.y);
                        }
                        st2(y + c0 + 2 * q, yv);
                        v[0] += (double)rtv[u].x * (double)yv.x;
                        v[0] += (double)rtv[u].y * (double)yv.y;
                    }
                }
            }
        } else {
        for (int base = threadIdx.x; base < cnt; base += U * blockDim.x) {
            Row7<T> rw[U];
            int jr[U];
            T rtv[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int c = base + u * blockDim.x;
                if (c < cnt) {
                    load_row7<T, T, MIXED>(d, a, x, c0 + c, rw[u], &jr[u]);
                    rtv[u] = rt[c0 + c];
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int c = base + u * blockDim.x;
                if (c < cnt) {
                    T yv = dot_row7<T, MIXED>(rw[u], d.do_k);
                    if (jr[u] >= d.jmax2) yv = T(0);
                    if (defl) yv = yv + (T)(cp * (double)d.defl_az[c0 + c]);
                    y[c0 + c] = yv;
                    v[0] += (double)rtv[u] * (double)yv;
                }
            }
        }
        }
        tile_partial<1>(b, d, tl.idx, v);
        run_add<1>(b, run, tl.sys, fin);
    }
    run_close<1>(b, run, fin);
}

// S = R - alpha*V and Snorm (model/leq_bicgs.f:365-375); deflated mixed systems
// also form c_s = z^T S / z^T A z.
template <typename T, bool MIXED>
__global__ void __launch_bounds__(256, 4) k_s_update(BatchView b)
{
    constexpr int U2 = Batch<T>::STREAM / 2;
    constexpr int NV = MIXED ? 2 : 1;
    TileRun run{-1, 0};
    auto fin = [&](SysState &st, const double(&tot)[NV]) {
        st.snorm = sqrt(tot[0]);
        if (MIXED)
            st.snorm_exit = (st.snorm <= 0.1 * st.tol * st.outer_rnorm0) ? 1 : 0;
        else
            st.snorm_exit = (!st.icheck && st.snorm <= DBL_EPSILON) ? 1 : 0;  // TOLMIN = EPSILON(ONE); none
                                                                              // with MINIMIZE_DOTPRODUCTS
        if (MIXED && st.defl) st.defl_cs = tot[NV - 1] / st.defl_e;
    };
    for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
        const Tile tl = b.tiles[t];
        const SysDev &d = b.sys[tl.sys];
        SysState &st = b.st[tl.sys];
        if (!gate_ok(st, G_INNER)) continue;
        const int64_t c0 = (int64_t)tl.idx * TILE_CELLS;
        const int cnt = (int)min((int64_t)TILE_CELLS, cells<T>(d) - c0);
        const T alpha = (T)st.alpha;
        const T *__restrict__ r = vec<T>(d, V_R) + c0;
        const T *__restrict__ vv = vec<T>(d, V_V) + c0;
        T *__restrict__ s = vec<T>(d, V_S) + c0;
        const bool defl = MIXED && st.defl;
        double v[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) v[k] = 0.0;
        const int np = cnt >> 1;
        for (int base = threadIdx.x; base < np; base += U2 * blockDim.x) {
            vec2_t<T> rv[U2], wv[U2];
#pragma unroll
            for (int u = 0; u < U2; ++u) {
                const int q = base + u * blockDim.x;
                if (q < np) {
                    rv[u] = ld2(r + 2 * q);
                    wv[u] = ld2(vv + 2 * q);
                }
            }
#pragma unroll
            for (int u = 0; u < U2; ++u) {
                const int q = base + u * blockDim.x;
                if (q < np) {
                    const T s0 = rv[u].x - alpha * wv[u].x, s1 = rv[u].y - alpha * wv[u].y;
                    st2(s + 2 * q, mk2<T>(s0, s1));
                    v[0] += (double)s0 * (double)s0;
                    v[0] += (double)s1 * (double)s1;
                    if (defl) v[NV - 1] += zdot2<T>(d.defl_z, c0 + 2 * q, mk2<T>(s0, s1));
                }
            }
        }
        if ((cnt & 1) && threadIdx.x == 0) {
            const int c = cnt - 1;
            const T sv = r[c] - alpha * vv[c];
            s[c] = sv;
            v[0] += (double)sv * (double)sv;
            if (defl && d.defl_z[c0 + c]) v[NV - 1] += (double)sv;
        }
        tile_partial<NV>(b, d, tl.idx, v);
        run_add<NV>(b, run, tl.sys, fin);
    }
    run_close<NV>(b, run, fin);
}

// T = A*Shat, omega = (T,S)/(T,T) with (T,T) = 0 -> SMALL_NUMBER (model/leq_bicgs.f:409-427).
template <typename T, bool MIXED, bool PAIR>
__global__ void __launch_bounds__(256) k_matvec_omega(BatchView b, int src)
{
    constexpr int U = 2;  // one-cell rows: two cells per thread and pass (80 registers in FP32)
    constexpr int UP = 1;  // one cell pair per thread and pass: fewer registers, more resident warps
    TileRun run{-1, 0};
    auto fin = [&](SysState &st, const double(&tot)[2]) {
        double txt = tot[1];
        if (txt == 0.0) txt = 1.0e-15;  // SMALL_NUMBER
        st.omega = tot[0] / txt;
    };
    for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
        const Tile tl = b.tiles[t];
        const SysDev &d = b.sys[tl.sys];
        SysState &st = b.st[tl.sys];
        if (!gate_ok(st, G_INNER_NOSNORM) || pair_rows<T>(d) != PAIR) continue;
        const int64_t c0 = (int64_t)tl.idx * TILE_CELLS;
        const int cnt = (int)min((int64_t)TILE_CELLS, cells<T>(d) - c0);
        const T *__restrict__ a = diag_base<T>(d);
        const T *__restrict__ x = vec<T>(d, src);
        const T *__restrict__ s = vec<T>(d, V_S);
        T *__restrict__ y = vec<T>(d, V_T);
        double v[2] = {0.0, 0.0};
        // deflated mixed systems: T = A (Shat + c_s z) = A Shat + c_s A z
        const bool defl = MIXED && st.defl;
        const double cs = defl ? st.defl_cs : 0.0;
        if constexpr (PAIR) {
            const int np = cnt >> 1;
            for (int base = threadIdx.x; base < np; base += UP * blockDim.x) {
                Pair7<T> rw[UP];
                int jr[UP];
                vec2_t<T> sv[UP];
#pragma unroll
                for (int u = 0; u < UP; ++u) {
                    const int q = base + u * blockDim.x;
                    if (q < np) {
                        load_pair7<T, MIXED>(d, a, x, c0 + 2 * q, rw[u], &jr[u]);
                        sv[u] = ld2(s + c0 + 2 * q);
                    }
                }
#pragma unroll
                for (int u = 0; u < UP; ++u) {
                    const int q = base + u * blockDim.x;
                    if (q < np) {
                        vec2_t<T> yv = dot_pair7<T, MIXED>(rw[u], d.do_k);
                        if (jr[u] >= d.jmax2) yv.x = T(0);  // pad cells of the padded FP32 arrays
                        if (jr[u] + 1 >= d.jmax2) yv.y = T(0);
                        if (defl) {
                            const float2 az = ld2(d.defl_az + c0 + 2 * q);
                            yv.x = yv.x + (T)(cs * (double)az.x);
                            yv.y = yv.y + (T)(cs * (double)az.y);
                        }
                        st2(y + c0 + 2 * q, yv);
                        v[0] += (double)yv.x * (double)sv[u].x;
                        v[1] += (double)yv.x * (double)yv.x;
                        v[0] += (double)yv.y * (double)sv[u].y;
                        v[1] += (double)yv.y * (double)yv.y;
                    }
                }
            }
        } else {
        for (int base = threadIdx.x; base < cnt; base += U * blockDim.x) {
            Row7<T> rw[U];
            int jr[U];
            T sv[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int c = base + u * blockDim.x;
                if (c < cnt) {
                    load_row7<T, T, MIXED>(d, a, x, c0 + c, rw[u], &jr[u]);
                    sv[u] = s[c0 + c];
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int c = base + u * blockDim.x;
                if (c < cnt) {
                    T yv = dot_row7<T, MIXED>(rw[u], d.do_k);
                    if (jr[u] >= d.jmax2) yv = T(0);
                    if (defl) yv = yv + (T)(cs * (double)d.defl_az[c0 + c]);
                    y[c0 + c] = yv;
                    v[0] += (double)yv * (double)sv[u];
                    v[1] += (double)yv * (double)yv;
                }
            }
        }
        }
        tile_partial<2>(b, d, tl.idx, v);
        run_add<2>(b, run, tl.sys, fin);
    }
    run_close<2>(b, run, fin);
}

// ------------------------------------------------------------------ staged FP32 matvec
// The mixed form's V = A*Phat with alpha (KIND 0) and T = A*Shat with omega
// (KIND 1), with the operands streamed into shared memory by bulk copies of the
// Tensor Memory Accelerator (cp.async.bulk, completion counted on an mbarrier).
// One producer warp fills a ring of MV_STAGES stages of MV_CELLS cells; the
// MV_THREADS consumer threads compute the oldest stage and hand its slot back
// through a second mbarrier, so the bytes in flight per SM no longer depend on
// the registers each thread holds, and the producer's bookkeeping (tile, state
// and system loads) overlaps the consumers' work.  A stage holds the six
// off-diagonals, the row sums (defect form), x and the reduction's second vector
// (Rtilde or S); with WIN also x one line (i-1, i+1) and one plane (k-1, k+1)
// away.  Other neighbours come from global memory.  Consumer thread t owns cells
// 2t and 2t+1 of every stage, the cells it owns in k_matvec_alpha /
// k_matvec_omega's pair form, in the same order, with the same roundings: the
// products and the partial sums are the same bits.
constexpr int MV_THREADS = 256;           // consumer threads
constexpr int MV_BLOCK = MV_THREADS + 32; // and one producer warp
// Shapes of the ring (option staged_matvec): whether x's line / plane windows are
// staged, cells per stage, stages, resident blocks per SM.  Larger stages (1024
// cells x 3, 2048 x 3, 1024 x 6) ran slower on 256^3 (10.3, 15.6, 16.8 ms of
// matvecs per solve against 9.2): resident consumer warps, not the number of
// copies, bound the kernel, and three blocks per SM is the register limit.
template <int CFG>
struct MvCfg;
template <>
struct MvCfg<1> {
    static constexpr bool WIN = true;
    static constexpr int CELLS = 512, STAGES = 4, BPS = 2;
};
template <>
struct MvCfg<2> {
    static constexpr bool WIN = false;
    static constexpr int CELLS = 512, STAGES = 4, BPS = 3;
};
enum : int { MA_KM = 0, MA_JM, MA_IM, MA_DEF, MA_IP, MA_JP, MA_KP, MA_X, MA_W, MA_XIM, MA_XIP, MA_XKM, MA_XKP };

template <bool WIN>
__host__ __device__ constexpr int mv_arrays() { return WIN ? 13 : 9; }

// One stage of the ring: its cells and, copied once per tile by the producer,
// what the consumers need of the system (shared-memory reads instead of loads
// through the system table).
struct MvMeta {
    int sys;   // -1: no more work
    int tile;  // tile index within the system
    int cnt;   // cells of this stage (0: a tile past the FP32 arrays' end)
    int last;  // the tile's last stage: its partial sum follows
    int64_t c; // first cell
    const float *x;   // the product's input
    float *y;         // its output
    const float *az;  // deflated systems: A z (else null)
    double cz;        // deflated systems: c_p (alpha) or c_s (omega)
    int64_t np;       // cells of the padded arrays
    FastDiv div_jp, div_i;
    int jp, imax2, jmax2, kmax2, cyc, do_k;
};

template <int CFG>
constexpr size_t mv_smem()
{
    using C = MvCfg<CFG>;
    return (size_t)C::STAGES * mv_arrays<C::WIN>() * C::CELLS * sizeof(float) + 2 * C::STAGES * sizeof(uint64_t) +
           C::STAGES * sizeof(MvMeta);
}

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *mb, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(mb)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t *mb, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(mb)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *mb)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_addr(mb)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *mb, unsigned parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(mb)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Waits for the phase of `parity` to complete; false after about two seconds.
__device__ __forceinline__ bool mbar_wait(uint64_t *mb, unsigned parity)
{
    const long long t0 = clock64();
    while (!mbar_try_wait(mb, parity))
        if (clock64() - t0 > (1LL << 32)) return false;
    return true;
}
// global -> shared bulk copy; addresses 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *mb)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(mb))
                 : "memory");
}
// OR of v over the consumer threads (named barrier 1)
__device__ __forceinline__ bool consumers_or(bool v)
{
    uint32_t r;
    asm volatile("{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.or.pred q, 1, %2, p;\n selp.u32 %0, 1, 0, q;\n}\n"
                 : "=r"(r)
                 : "r"((uint32_t)v), "n"(MV_THREADS)
                 : "memory");
    return r != 0;
}

template <int KIND, int CFG>
__global__ void __launch_bounds__(MV_BLOCK, MvCfg<CFG>::BPS) k_matvec_staged(BatchView b, int src)
{
    constexpr bool WIN = MvCfg<CFG>::WIN;
    constexpr int MV_CELLS = MvCfg<CFG>::CELLS;
    constexpr int MV_STAGES = MvCfg<CFG>::STAGES;
    constexpr int NA = mv_arrays<WIN>();
    constexpr int NV = KIND == 0 ? 1 : 2;
    extern __shared__ __align__(128) unsigned char mv_smem[];
    float *buf = reinterpret_cast<float *>(mv_smem);
    uint64_t *full = reinterpret_cast<uint64_t *>(mv_smem + (size_t)MV_STAGES * NA * MV_CELLS * sizeof(float));
    uint64_t *empty = full + MV_STAGES;
    MvMeta *meta = reinterpret_cast<MvMeta *>(empty + MV_STAGES);
    const int gate = KIND == 0 ? G_INNER : G_INNER_NOSNORM;
    const int wid = KIND == 0 ? V_RT : V_S;
    const int yid = KIND == 0 ? V_V : V_T;
    if (threadIdx.x == 0) {
        for (int q = 0; q < MV_STAGES; ++q) {
            mbar_init(full + q, 1);
            mbar_init(empty + q, MV_THREADS / 32);
        }
        mbar_fence_init();
    }
    __syncthreads();

    if (threadIdx.x >= MV_THREADS) {
        // ---- producer: the block's tiles t = blockIdx.x + m*gridDim.x of the systems
        // in this reduction, MV_CELLS cells a stage
        if (threadIdx.x != MV_THREADS) return;
        int pt = blockIdx.x, psub = 0, cur = -1;
        MvMeta tm;  // the current tile's system fields
        tm.sys = -1;
        int64_t t0 = 0, tend = 0, c2 = 0;
        const float *a = nullptr, *def = nullptr, *w = nullptr;
        int last_s[MV_STAGES];
        for (int q = 0; q < MV_STAGES; ++q) last_s[q] = -1;
        for (int s = 0;; ++s) {
            const int slot = s % MV_STAGES;
            if (s >= MV_STAGES && !mbar_wait(empty + slot, (unsigned)(s / MV_STAGES - 1) & 1u)) {
                // the consumers gave up: the copies still in flight, again bounded
                for (int q = 0; q < MV_STAGES; ++q)
                    if (last_s[q] >= 0) mbar_wait(full + q, (unsigned)(last_s[q] / MV_STAGES) & 1u);
                return;
            }
            MvMeta m = tm;
            m.sys = -1;
            m.tile = 0;
            m.cnt = 0;
            m.last = 0;
            m.c = 0;
            while (pt < b.ntiles) {
                if (pt != cur) {
                    const Tile tl = b.tiles[pt];
                    const SysState &st = b.st[tl.sys];
                    if (!gate_ok(st, gate)) {
                        pt += gridDim.x;
                        psub = 0;
                        continue;
                    }
                    const SysDev &d = b.sys[tl.sys];
                    cur = pt;
                    tm.sys = tl.sys;
                    tm.tile = tl.idx;
                    tm.x = vec<float>(d, src);
                    tm.y = vec<float>(d, yid);
                    tm.az = st.defl ? d.defl_az : nullptr;
                    tm.cz = st.defl ? (KIND == 0 ? st.defl_cp : st.defl_cs) : 0.0;
                    tm.np = d.np;
                    tm.div_jp = d.div_jp;
                    tm.div_i = d.div_i;
                    tm.jp = d.jp;
                    tm.imax2 = d.imax2;
                    tm.jmax2 = d.jmax2;
                    tm.kmax2 = d.kmax2;
                    tm.cyc = d.cyc;
                    tm.do_k = d.do_k;
                    a = d.a32;
                    def = d.defect;
                    w = vec<float>(d, wid);
                    c2 = (int64_t)d.jp * d.imax2;
                    t0 = (int64_t)tl.idx * TILE_CELLS;
                    tend = min(t0 + TILE_CELLS, d.np);
                }
                m = tm;
                m.c = t0 + (int64_t)psub * MV_CELLS;
                m.cnt = (int)max((int64_t)0, min((int64_t)MV_CELLS, tend - m.c));
                m.last = m.c + MV_CELLS >= tend;
                if (m.last) {
                    pt += gridDim.x;
                    psub = 0;
                } else {
                    ++psub;
                }
                break;
            }
            meta[slot] = m;
            if (m.cnt == 0) {
                mbar_arrive(full + slot);
                if (m.sys < 0) return;
                continue;
            }
            // array q holds cells [c + shift, c + shift + cnt) of its source, clipped
            // to the source's [0, np)
            float *sb = buf + (size_t)slot * NA * MV_CELLS;
            const int64_t c = m.c, cnt = m.cnt, np = m.np, c1 = m.jp;
            const float *x = m.x;
            const float *srcs[NA];
            int64_t shift[NA];
            for (int q = 0; q < NA; ++q) srcs[q] = nullptr, shift[q] = 0;
            srcs[MA_JM] = a + 1 * np;
            srcs[MA_IM] = a + 2 * np;
            srcs[MA_DEF] = def;
            srcs[MA_IP] = a + 4 * np;
            srcs[MA_JP] = a + 5 * np;
            srcs[MA_X] = x;
            srcs[MA_W] = w;
            if (m.do_k) {
                srcs[MA_KM] = a + 0 * np;
                srcs[MA_KP] = a + 6 * np;
            }
            if constexpr (WIN) {
                srcs[MA_XIM] = x, shift[MA_XIM] = -c1;
                srcs[MA_XIP] = x, shift[MA_XIP] = c1;
                if (m.do_k) {
                    srcs[MA_XKM] = x, shift[MA_XKM] = -c2;
                    srcs[MA_XKP] = x, shift[MA_XKP] = c2;
                }
            }
            unsigned bytes = 0;
#pragma unroll
            for (int q = 0; q < NA; ++q) {
                const int64_t lo = max(c + shift[q], (int64_t)0), hi = min(c + shift[q] + cnt, np);
                if (srcs[q] && hi > lo) bytes += (unsigned)((hi - lo) * sizeof(float));
            }
            mbar_expect_tx(full + slot, bytes);
#pragma unroll
            for (int q = 0; q < NA; ++q) {
                const int64_t lo = max(c + shift[q], (int64_t)0), hi = min(c + shift[q] + cnt, np);
                if (srcs[q] && hi > lo)
                    bulk_g2s(sb + q * MV_CELLS + (lo - c - shift[q]), srcs[q] + lo, (unsigned)((hi - lo) * sizeof(float)),
                             full + slot);
            }
            last_s[slot] = s;
        }
    }

    // ---- consumers
    auto fin = [&](SysState &st, const double(&tot)[NV]) {
        if constexpr (KIND == 0) {
            st.alpha = st.rho / tot[0];
        } else {
            double txt = tot[NV - 1];
            if (txt == 0.0) txt = 1.0e-15;  // SMALL_NUMBER
            st.omega = tot[0] / txt;
        }
    };
    TileRun run{-1, 0};
    double v[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = 0.0;
    for (int s = 0;; ++s) {
        const int slot = s % MV_STAGES;
        const bool ok = mbar_wait(full + slot, (unsigned)(s / MV_STAGES) & 1u);
        if (consumers_or(!ok)) {  // the same answer in every consumer thread
            if (threadIdx.x == 0) {
                const int sys = meta[slot].sys;
                atomicOr(&b.st[sys >= 0 && sys < b.nsys ? sys : 0].err, 4);
            }
            return;
        }
        const MvMeta &m = meta[slot];
        const int sys = m.sys;
        if (sys < 0) break;
        const int tile = m.tile, last = m.last;
        for (int u = 0; u < MV_CELLS / (2 * MV_THREADS); ++u) {
        const int l = 2 * (threadIdx.x + MV_THREADS * u);
        if (l < m.cnt) {
            const float *sb = buf + (size_t)slot * NA * MV_CELLS;
            const float *x = m.x;
            const int64_t p = m.c + l;
            const int jp = m.jp, imax2 = m.imax2, jmax2 = m.jmax2;
            const uint32_t line = fdiv((uint32_t)p, m.div_jp);
            const int j = (int)((uint32_t)p - line * (uint32_t)jp);
            const uint32_t kk = fdiv(line, m.div_i);
            const int k = (int)kk, i = (int)(line - kk * (uint32_t)imax2);
            const int64_t c1 = jp, c2 = (int64_t)jp * imax2;
            const float2 xc = *reinterpret_cast<const float2 *>(sb + MA_X * MV_CELLS + l);
            // x at an i or k neighbour (the pair shares i and k): the cells themselves,
            // the staged window, or global memory (in bounds for every cell's offset)
            auto nb2 = [&](int arr, int64_t off, int64_t win) -> float2 {
                if (off == 0) return xc;
                if constexpr (WIN)
                    if (off == win) return *reinterpret_cast<const float2 *>(sb + arr * MV_CELLS + l);
                return __ldg(reinterpret_cast<const float2 *>(x + p + off));
            };
            // x at cell p + off of the stage's own cells, or from global memory
            auto xat = [&](int64_t off) -> float {
                const int64_t t = l + off;
                if (t >= 0 && t < m.cnt) return sb[MA_X * MV_CELLS + t];
                const int64_t g = p + off;
                return (g >= 0 && g < m.np) ? __ldg(x + g) : 0.0f;  // out of range only for pad cells
            };
            float xjm0, xjm1, xjp0, xjp1;
            int64_t im, ip, km = 0, kp = 0;
            if (m.cyc == 0) {  // clamped neighbours (model/set_increments.f:80-109)
                xjm0 = j > 0 ? xat(-1) : xc.x;
                xjm1 = xc.x;
                xjp0 = j < jmax2 - 1 ? xc.y : xc.x;
                xjp1 = j + 1 < jmax2 - 1 ? xat(2) : xc.y;
                im = i > 0 ? -c1 : 0;
                ip = i < imax2 - 1 ? c1 : 0;
                if (m.do_k) {
                    km = k > 0 ? -c2 : 0;
                    kp = k < m.kmax2 - 1 ? c2 : 0;
                }
            } else {
                const bool cj = (m.cyc & 2) != 0;
                const int64_t o0 = inc_m(j, jmax2, cj), o1 = inc_m(j + 1, jmax2, cj);
                const int64_t o2 = inc_p(j, jmax2, cj), o3 = inc_p(j + 1, jmax2, cj);
                xjm0 = o0 == 0 ? xc.x : xat(o0);
                xjm1 = o1 == 0 ? xc.y : xat(1 + o1);
                xjp0 = o2 == 0 ? xc.x : xat(o2);
                xjp1 = o3 == 0 ? xc.y : xat(1 + o3);
                im = inc_m(i, imax2, m.cyc & 1) * c1;
                ip = inc_p(i, imax2, m.cyc & 1) * c1;
                if (m.do_k) {
                    km = inc_m(k, m.kmax2, m.cyc & 4) * c2;
                    kp = inc_p(k, m.kmax2, m.cyc & 4) * c2;
                }
            }
            const float2 xim = nb2(MA_XIM, im, -c1);
            const float2 xip = nb2(MA_XIP, ip, c1);
            const float2 ajm = *reinterpret_cast<const float2 *>(sb + MA_JM * MV_CELLS + l);
            const float2 aim = *reinterpret_cast<const float2 *>(sb + MA_IM * MV_CELLS + l);
            const float2 rs = *reinterpret_cast<const float2 *>(sb + MA_DEF * MV_CELLS + l);
            const float2 aip = *reinterpret_cast<const float2 *>(sb + MA_IP * MV_CELLS + l);
            const float2 ajp = *reinterpret_cast<const float2 *>(sb + MA_JP * MV_CELLS + l);
            // dot_pair7's defect form, operand for operand
            float u = dterm0(ajm.x, xjm0, xc.x);
            float t = dterm0(ajm.y, xjm1, xc.y);
            u = dterm(u, aim.x, xim.x, xc.x);
            t = dterm(t, aim.y, xim.y, xc.y);
            u = dcentre(u, rs.x, xc.x);
            t = dcentre(t, rs.y, xc.y);
            u = dterm(u, aip.x, xip.x, xc.x);
            t = dterm(t, aip.y, xip.y, xc.y);
            u = dterm(u, ajp.x, xjp0, xc.x);
            t = dterm(t, ajp.y, xjp1, xc.y);
            if (m.do_k) {
                const float2 xkm = nb2(MA_XKM, km, -c2);
                const float2 xkp = nb2(MA_XKP, kp, c2);
                const float2 akm = *reinterpret_cast<const float2 *>(sb + MA_KM * MV_CELLS + l);
                const float2 akp = *reinterpret_cast<const float2 *>(sb + MA_KP * MV_CELLS + l);
                u = dterm(u, akm.x, xkm.x, xc.x);
                t = dterm(t, akm.y, xkm.y, xc.y);
                u = dterm(u, akp.x, xkp.x, xc.x);
                t = dterm(t, akp.y, xkp.y, xc.y);
            }
            if (j >= jmax2) u = 0.0f;  // pad cells of the padded FP32 arrays
            if (j + 1 >= jmax2) t = 0.0f;
            const float2 wv = *reinterpret_cast<const float2 *>(sb + MA_W * MV_CELLS + l);
            if (m.az) {  // deflated systems: A (Phat + c z) = A Phat + c A z
                const float2 az = ld2(m.az + p);
                u = u + (float)(m.cz * (double)az.x);
                t = t + (float)(m.cz * (double)az.y);
            }
            st2(m.y + p, mk2<float>(u, t));
            if constexpr (KIND == 0) {
                v[0] += (double)wv.x * (double)u;
                v[0] += (double)wv.y * (double)t;
            } else {
                v[0] += (double)u * (double)wv.x;
                v[NV - 1] += (double)u * (double)u;
                v[0] += (double)t * (double)wv.y;
                v[NV - 1] += (double)t * (double)t;
            }
        }
        }
        __syncwarp();
        if ((threadIdx.x & 31) == 0) mbar_arrive(empty + slot);  // this warp is done with the slot
        if (last) {
            tile_partial<NV, 1, MV_THREADS>(b, b.sys[sys], tile, v);
            run_add<NV, 1, MV_THREADS>(b, run, sys, fin);
#pragma unroll
            for (int q = 0; q < NV; ++q) v[q] = 0.0;
        }
    }
    run_close<NV, 1, MV_THREADS>(b, run, fin);
}

// X += alpha*Phat + omega*Shat; R = S - omega*T; Rnorm; next rho
// (model/leq_bicgs.f:432-460 and :318 of the following iteration).
__device__ inline void fin_xr_ref(SysState &s, double rr, double rtr)
{
    if (s.snorm_exit) {  // :375-395
        s.ier = 0;
        s.exit_kind = EX_SNORM;
        s.status = ST_DONE;
        return;
    }
    // with MINIMIZE_DOTPRODUCTS Rnorm is formed and tested every icheck-th
    // iteration only (model/leq_bicgs.f:439; LEQ_BICGSt: every fifth, leq_bicgst.f:514)
    if (!s.icheck || s.iter % s.icheck == 0) {
        s.rnorm = sqrt(rr);
        if (s.rnorm <= s.tol * s.rnorm0) {
            s.iter_tot_add = s.iter + 1;
            s.ier = 0;
            s.exit_kind = EX_RNORM;
            s.status = ST_DONE;
            return;
        }
    }
    s.iter += 1;
    s.i += 1;
    if (s.i > s.itmax) {
        final_logic(s, false);
        return;
    }
    s.beta = (rtr / s.rho) * (s.alpha / s.omega);
    s.rho_prev = s.rho;
    s.rho = rtr;
    if (rtr == 0.0) {
        s.ier = -2;
        s.exit_kind = EX_RHO0;
        s.status = ST_DONE;
    }
}

// Mixed form (FP32 BiCGSTAB with reliable updates): once the FP32 recursive
// residual has dropped by inner_tol against the largest value since the last
// update, or looks converged, the system goes to the FP64 step, which folds the
// FP32 correction into x and replaces the residual by the true one.
__device__ inline void fin_xr_inner(SysState &s, double rr, double rtr)
{
    s.inner_total += 1;
    s.inner_first = 0;
    if (s.snorm_exit) {  // omega was not formed: restart after the update
        s.phase = PH_OUTER;
        s.restart = 1;
        return;
    }
    const double rn = sqrt(rr);
    s.rnorm = rn;
    if (!(rn == rn)) {
        s.phase = PH_OUTER;
        s.restart = 1;
        return;
    }
    if (rn > s.maxr) s.maxr = rn;
    s.since_outer += 1;
    // deflated (near-singular) systems also replace the residual at a fixed
    // interval: their slow FP32 recurrence drifts from the true residual long
    // before it has dropped by inner_tol
    const bool due = s.defl && s.replace_every > 0 && s.since_outer >= s.replace_every;
    if (rn <= s.inner_tol * s.maxr || rn <= s.tol * s.outer_rnorm0 || s.inner_total >= s.itmax || due) {
        s.phase = PH_OUTER;
        return;
    }
    s.beta = (rtr / s.rho) * (s.alpha / s.omega);
    s.rho_prev = s.rho;
    s.rho = rtr;
    s.i += 1;
    if (rtr == 0.0 || s.omega == 0.0) {
        s.phase = PH_OUTER;
        s.restart = 1;
    }
}

// The mixed form accumulates x in the caller's VAR (natural layout) while its
// FP32 vectors are padded: the cells of padded pair p (p even) in VAR.
struct NatPair {
    int64_t c;     // natural cell of the pair's first element
    bool r0, r1;   // which of the two elements are cells (not pads)
};
__device__ __forceinline__ NatPair nat_pair(const SysDev &d, int64_t p)
{
    const uint32_t line = fdiv((uint32_t)p, d.div_jp);
    const int j = (int)(p - (int64_t)line * d.jp);
    return NatPair{(int64_t)line * d.jmax2 + j, j < d.jmax2, j + 1 < d.jmax2};
}

template <typename T, bool MIXED>
__global__ void __launch_bounds__(256) k_xr_update(BatchView b, int ph_id, int sh_id)
{
    constexpr int U2 = 1;  // one cell pair per thread and pass: 60-64 registers, 4 blocks per SM
    TileRun run{-1, 0};
    auto fin = [&](SysState &st, const double(&tot)[2]) {
        if (MIXED)
            fin_xr_inner(st, tot[0], tot[1]);
        else
            fin_xr_ref(st, tot[0], tot[1]);
    };
    for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
        const Tile tl = b.tiles[t];
        const SysDev &d = b.sys[tl.sys];
        SysState &st = b.st[tl.sys];
        if (!gate_ok(st, G_INNER)) continue;
        const int64_t c0 = (int64_t)tl.idx * TILE_CELLS;
        const int cnt = (int)min((int64_t)TILE_CELLS, cells<T>(d) - c0);
        // FP64 drop-in: X is VAR.  Mixed form: the solution is accumulated in FP64
        // every iteration (x64 += alpha*Phat + omega*Shat with FP64 scalars), in
        // VAR's own layout (nat_pair maps the padded pairs onto it).
        using X_T = typename std::conditional<MIXED, double, T>::type;
        X_T *__restrict__ x =
            MIXED ? reinterpret_cast<X_T *>(d.x64[0]) : reinterpret_cast<X_T *>(vec<T>(d, V_X)) + c0;
        auto xload = [&](int q) -> vec2_t<X_T> {
            if constexpr (MIXED) {
                const NatPair np2 = nat_pair(d, c0 + 2 * q);
                return mk2<X_T>(np2.r0 ? x[np2.c] : X_T(0), np2.r1 ? x[np2.c + 1] : X_T(0));
            } else {
                return ld2(x + 2 * q);
            }
        };
        auto xstore = [&](int q, const vec2_t<X_T> &v) {
            if constexpr (MIXED) {
                const NatPair np2 = nat_pair(d, c0 + 2 * q);
                if (np2.r0) x[np2.c] = v.x;
                if (np2.r1) x[np2.c + 1] = v.y;
            } else {
                st2(x + 2 * q, v);
            }
        };
        const X_T alpha = (X_T)st.alpha;
        const T *__restrict__ ph = vec<T>(d, ph_id) + c0;
        double v[2] = {0.0, 0.0};
        const int np = cnt >> 1;
        // deflated mixed systems: Phat + c_p z and Shat + c_s z, so x also gains
        // (alpha c_p + omega c_s) on the coupled rows
        const bool defl = MIXED && st.defl;
        const unsigned char *__restrict__ zr = defl ? d.defl_z + c0 : nullptr;
        if (st.snorm_exit) {
            const X_T wz = defl ? (X_T)(st.alpha * st.defl_cp) : X_T(0);
            for (int base = threadIdx.x; base < np; base += U2 * blockDim.x) {
                vec2_t<X_T> xv[U2];
                vec2_t<T> pv[U2];
#pragma unroll
                for (int u = 0; u < U2; ++u) {
                    const int q = base + u * blockDim.x;
                    if (q < np) {
                        xv[u] = xload(q);
                        pv[u] = ld2(ph + 2 * q);
                    }
                }
#pragma unroll
                for (int u = 0; u < U2; ++u) {
                    const int q = base + u * blockDim.x;
                    if (q < np) {
                        vec2_t<X_T> xn = mk2<X_T>(xv[u].x + alpha * (X_T)pv[u].x, xv[u].y + alpha * (X_T)pv[u].y);
                        if (defl) {
                            const uchar2 zz = *reinterpret_cast<const uchar2 *>(zr + 2 * q);
                            if (zz.x) xn.x = xn.x + wz;
                            if (zz.y) xn.y = xn.y + wz;
                        }
                        xstore(q, xn);
                    }
                }
            }
            if (!MIXED && (cnt & 1) && threadIdx.x == 0) x[cnt - 1] = x[cnt - 1] + alpha * (X_T)ph[cnt - 1];
        } else {
            const X_T omega = (X_T)st.omega;
            const X_T wz = defl ? (X_T)(st.alpha * st.defl_cp + st.omega * st.defl_cs) : X_T(0);
            const T omega_t = (T)st.omega;
            const T *__restrict__ sh = vec<T>(d, sh_id) + c0;
            const T *__restrict__ s = vec<T>(d, V_S) + c0;
            const T *__restrict__ tv = vec<T>(d, V_T) + c0;
            const T *__restrict__ rt = vec<T>(d, V_RT) + c0;
            T *__restrict__ r = vec<T>(d, V_R) + c0;
            for (int base = threadIdx.x; base < np; base += U2 * blockDim.x) {
                vec2_t<X_T> xv[U2];
                vec2_t<T> pv[U2], hv[U2], sv[U2], tw[U2], rtv[U2];
#pragma unroll
                for (int u = 0; u < U2; ++u) {
                    const int q = base + u * blockDim.x;
                    if (q < np) {
                        xv[u] = xload(q);
                        pv[u] = ld2(ph + 2 * q);
                        hv[u] = ld2(sh + 2 * q);
                        sv[u] = ld2(s + 2 * q);
                        tw[u] = ld2(tv + 2 * q);
                        rtv[u] = ld2(rt + 2 * q);
                    }
                }
#pragma unroll
                for (int u = 0; u < U2; ++u) {
                    const int q = base + u * blockDim.x;
                    if (q < np) {
                        vec2_t<X_T> xn = mk2<X_T>(xv[u].x + alpha * (X_T)pv[u].x + omega * (X_T)hv[u].x,
                                                  xv[u].y + alpha * (X_T)pv[u].y + omega * (X_T)hv[u].y);
                        if (defl) {
                            const uchar2 zz = *reinterpret_cast<const uchar2 *>(zr + 2 * q);
                            if (zz.x) xn.x = xn.x + wz;
                            if (zz.y) xn.y = xn.y + wz;
                        }
                        xstore(q, xn);
                        const T r0 = sv[u].x - omega_t * tw[u].x, r1 = sv[u].y - omega_t * tw[u].y;
                        st2(r + 2 * q, mk2<T>(r0, r1));
                        v[0] += (double)r0 * (double)r0;
                        v[1] += (double)rtv[u].x * (double)r0;
                        v[0] += (double)r1 * (double)r1;
                        v[1] += (double)rtv[u].y * (double)r1;
                    }
                }
            }
            if (!MIXED && (cnt & 1) && threadIdx.x == 0) {
                const int c = cnt - 1;
                x[c] = x[c] + alpha * (X_T)ph[c] + omega * (X_T)sh[c];
                const T rv = s[c] - omega_t * tv[c];
                r[c] = rv;
                v[0] += (double)rv * (double)rv;
                v[1] += (double)rt[c] * (double)rv;
            }
        }
        tile_partial<2>(b, d, tl.idx, v);
        run_add<2>(b, run, tl.sys, fin);
    }
    run_close<2>(b, run, fin);
}

// ------------------------------------------------------------------ mixed form: reliable update
// x <- x + d in FP64, r = b - A x in FP64 with the FP64 A; the FP32 residual is
// replaced by the true one.  The Krylov process continues (P and Rtilde kept,
// beta formed from the replaced residual) unless a restart was asked for.
__device__ inline void fin_outer(SysState &s, double rr, double rtr32)
{
    const double rn = sqrt(rr);
    const bool fresh = (s.outer_steps == 0) || s.restart;
    if (s.outer_steps == 0) {
        s.outer_rnorm0 = rn;
        s.best = rn;
    }
    s.outer_rnorm = rn;
    s.outer_steps += 1;
    s.rnorm = rn;
    s.rnorm0 = s.outer_rnorm0;
    if (rn <= s.tol * s.outer_rnorm0) {
        s.iter = s.inner_total;
        s.iter_tot_add = s.inner_total + 1;
        s.ier = 0;
        s.exit_kind = EX_RNORM;
        s.status = ST_DONE;
        return;
    }
    // guard: FP32 iterations that diverge or stall on a (near-)singular operator
    // hand the system to an FP64 re-solve instead of returning a worse answer.
    // A deflated system's residual plateaus for hundreds of iterations (as the
    // FP64 drop-in's does on it) and is replaced at a fixed interval, so its
    // stall window is 400 iterations and its growth limit 1e4.
    if (rn < 0.9 * s.best) {
        s.best = rn;
        s.stall = 0;
    } else {
        s.stall += 1;
    }
    int stall_limit = s.stall_limit;
    double growth_limit = s.growth_limit;
    if (s.defl && s.replace_every > 0) {
        stall_limit = max(stall_limit, (400 + s.replace_every - 1) / s.replace_every);
        growth_limit = fmax(growth_limit, 1e4);
    }
    if (!(rn == rn) || rn > growth_limit * s.best || s.stall >= stall_limit) {
        s.exit_kind = EX_FALLBACK;
        s.ier = -20;
        s.status = ST_DONE;
        return;
    }
    // ITMAX spent without reaching TOL: the FP64 drop-in re-solves from the initial
    // guess and gives the verdict (the mixed form is never worse than FP64's)
    if (s.inner_total >= s.itmax) {
        s.exit_kind = EX_FALLBACK;
        s.ier = -20;
        s.status = ST_DONE;
        return;
    }
    // a deflated system whose true residual has risen restart_growth-fold above its
    // best: the FP32 Krylov process has drifted away from the FP64 residual, so it
    // restarts from the true residual (Rtilde = R, P = R) at the next update, the
    // stall window still bounding the restarts
    if (s.defl && !fresh && s.restart_growth > 0.0 && rn > s.restart_growth * s.best) {
        s.restart = 1;
        s.phase = PH_OUTER;
        return;
    }
    s.maxr = rn;
    s.inner_first = 1;
    s.since_outer = 0;
    s.snorm_exit = 0;
    s.phase = PH_INNER;
    if (fresh) {
        s.rho = rtr32;
        s.i = 1;
        s.restart = 0;
        if (!(rtr32 > 0.0)) {  // the FP32 copy of a nonzero FP64 residual vanished
            s.exit_kind = EX_FALLBACK;
            s.ier = -20;
            s.status = ST_DONE;
        }
        return;
    }
    s.beta = (rtr32 / s.rho) * (s.alpha / s.omega);
    s.rho_prev = s.rho;
    s.rho = rtr32;
    s.i += 1;
    if (rtr32 == 0.0 || !(s.beta == s.beta)) {  // breakdown: restart at the next update
        s.restart = 1;
        s.phase = PH_OUTER;
    }
}

// True when a tile this block visits belongs to a system that passes the gate.
// Every thread checks different tiles of the block's share, so a launch with
// nothing to do costs one round of loads instead of one per tile in turn.
__device__ __forceinline__ bool block_has_work(const BatchView &b, int gate)
{
    bool any = false;
    for (int t = blockIdx.x + threadIdx.x * gridDim.x; t < b.ntiles && !any; t += blockDim.x * gridDim.x)
        any = gate_ok(b.st[b.tiles[t].sys], gate);
    return __syncthreads_or(any) != 0;
}

__global__ void __launch_bounds__(256) k_outer_step(BatchView b)
{
    constexpr int U = 2;
    TileRun run{-1, 0};
    auto fin = [&](SysState &st, const double(&tot)[2]) { fin_outer(st, tot[0], tot[1]); };
    // most launches find no system due for a reliable update
    if (!block_has_work(b, G_OUTER)) return;
    for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
        const Tile tl = b.tiles[t];
        const SysDev &d = b.sys[tl.sys];
        SysState &st = b.st[tl.sys];
        if (!gate_ok(st, G_OUTER)) continue;
        const int64_t c0 = (int64_t)tl.idx * TILE_CELLS;
        const int cnt = (int)min((int64_t)TILE_CELLS, d.n - c0);
        const double *__restrict__ x = d.x64[0];
        const bool fresh = (st.outer_steps == 0) || st.restart;
        float *__restrict__ r32 = vec<float>(d, V_R);
        float *__restrict__ rt32 = vec<float>(d, V_RT);
        double v[2] = {0.0, 0.0};
        for (int base = threadIdx.x; base < cnt; base += U * blockDim.x) {
            Row7<double> rw[U];
            double bv[U];
            float rtv[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int c = base + u * blockDim.x;
                if (c < cnt) {
                    load_row7<double, double>(d, d.a64, x, c0 + c, rw[u]);
                    bv[u] = d.b64[c0 + c];
                    rtv[u] = fresh ? 0.f : rt32[padded(d, c0 + c)];
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int c = base + u * blockDim.x;
                if (c < cnt) {
                    const double rv = bv[u] - dot_row7<double>(rw[u], d.do_k);
                    const float rf = (float)rv;
                    const int64_t pc = padded(d, c0 + c);  // the FP32 vectors are padded
                    r32[pc] = rf;
                    const float rtf = fresh ? rf : rtv[u];
                    if (fresh) rt32[pc] = rf;
                    v[0] += rv * rv;
                    v[1] += (double)rtf * (double)rf;
                }
            }
        }
        tile_partial<2>(b, d, tl.idx, v);
        run_add<2>(b, run, tl.sys, fin);
    }
    run_close<2>(b, run, fin);
}

// ------------------------------------------------------------------ J-line half-sweeps
// Row r of the J-line at (i,k), as LEQ_IKSWEEP / LEQ_ISWEEP build it
// (model/leqsol_mod.f:891-905, :807-819): sub = A(-2), diag = A(0),
// super = A(2), rhs = B - A(-1)Var(i-1) - A(1)Var(i+1) [- A(-3)Var(k-1) - A(3)Var(k+1)],
// with CC(first) = EE(last) = 0.  Neighbours that clamp onto the cell itself read
// the cell's own value from before the sweep.
template <typename T>
struct LineCtx {
    const T *a;
    const T *rhs;
    const T *nb_im, *nb_ip, *nb_km, *nb_kp;  // already offset to the line base
    int64_t base, n;
    int L, do_k;
};

template <typename T>
__device__ __forceinline__ void line_row(const LineCtx<T> &x, int r, T &sub, T &dg, T &sup, T &f)
{
    const int64_t p = x.base + r;
    const int64_t n = x.n;
    sub = (r == 0) ? T(0) : x.a[1 * n + p];
    dg = x.a[3 * n + p];
    sup = (r == x.L - 1) ? T(0) : x.a[5 * n + p];
    T v = x.rhs[p] - x.a[2 * n + p] * x.nb_im[r];
    v = v - x.a[4 * n + p] * x.nb_ip[r];
    if (x.do_k) {
        v = v - x.a[0 * n + p] * x.nb_km[r];
        v = v - x.a[6 * n + p] * x.nb_kp[r];
    }
    f = v;
}

// DGTSV (NRHS = 1) on shared-memory rows 0..L-1: sub[r] couples row r to r-1,
// sup[r] couples row r to r+1.  Same pivoting and INFO as model/DGTSV.f:107-163, 231-246.
template <typename T>
__device__ int dgtsv_rows(int L, T *sub, T *dg, T *sup, T *f)
{
    // DL(i) = sub[i+1] (i = 0..L-2); DL is overwritten by the second super-diagonal.
    for (int i = 0; i < L - 1; ++i) {
        T dli = sub[i + 1];
        if (fabs(dg[i]) >= fabs(dli)) {
            if (dg[i] != T(0)) {
                const T fact = dli / dg[i];
                dg[i + 1] = dg[i + 1] - fact * sup[i];
                f[i + 1] = f[i + 1] - fact * f[i];
            } else {
                return i + 1;
            }
            if (i < L - 2) sub[i + 1] = T(0);
        } else {
            const T fact = dg[i] / dli;
            dg[i] = dli;
            const T temp = dg[i + 1];
            dg[i + 1] = sup[i] - fact * temp;
            if (i < L - 2) {
                sub[i + 1] = sup[i + 1];
                sup[i + 1] = -fact * sub[i + 1];
            }
            sup[i] = temp;
            const T tb = f[i];
            f[i] = f[i + 1];
            f[i + 1] = tb - fact * f[i + 1];
        }
    }
    if (dg[L - 1] == T(0)) return L;
    f[L - 1] = f[L - 1] / dg[L - 1];
    if (L > 1) f[L - 2] = (f[L - 2] - sup[L - 2] * f[L - 1]) / dg[L - 2];
    for (int i = L - 3; i >= 0; --i) f[i] = (f[i] - sup[i] * f[i + 1] - sub[i + 1] * f[i + 2]) / dg[i];
    return 0;
}

// DGTSV's INFO alone: the same interchanges and zero-pivot tests as dgtsv_rows on
// the matrix rows, no right-hand side (INFO does not depend on it).
template <typename T>
__device__ int dgtsv_info(int L, T *sub, T *dg, T *sup)
{
    for (int i = 0; i < L - 1; ++i) {
        T dli = sub[i + 1];
        if (fabs(dg[i]) >= fabs(dli)) {
            if (dg[i] != T(0)) {
                const T fact = dli / dg[i];
                dg[i + 1] = dg[i + 1] - fact * sup[i];
            } else {
                return i + 1;
            }
            if (i < L - 2) sub[i + 1] = T(0);
        } else {
            const T fact = dg[i] / dli;
            dg[i] = dli;
            const T temp = dg[i + 1];
            dg[i + 1] = sup[i] - fact * temp;
            if (i < L - 2) {
                sub[i + 1] = sup[i + 1];
                sup[i + 1] = -fact * sub[i + 1];
            }
            sup[i] = temp;
        }
    }
    return dg[L - 1] == T(0) ? L : 0;
}

__device__ __forceinline__ int find_sys(const int *prefix, int nsys, int item)
{
    int lo = 0, hi = nsys - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(prefix + mid) <= item)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// The line (i, k), 1-based, of slot q of a kind-0 wave (lines with (i+k) of the
// wave's parity, 3-D sweeps (i+k) odd first (model/leqsol_mod.f:497-509), 2-D
// sweeps i odd first (:382-391), i.e. (i+k) even with k = 1: the wave's parity is
// stated for 3-D and flipped for a 2-D system); false when the slot is past the
// system's lines or outside the wave's wrap level.
__device__ __forceinline__ bool wave_line(const SysDev &d, const WaveArgs &w, int q, int &i, int &k)
{
    k = (int)fdiv((uint32_t)q, d.div_h) + 1;
    const int slot = q - (k - 1) * d.half_lines;
    const int par = d.do_k ? w.par : (w.par ^ 1);
    const int i0 = (((1 + k) & 1) == par) ? 1 : 2;
    i = i0 + 2 * slot;
    bool valid = (k <= d.kmax2) && (i <= d.imax2);
    if (w.lvl > 0 && valid) valid = wrap_level(d, i, k) == w.lvl - 1;
    return valid;
}

struct LineJob {
    int item;
    int sidx;
    int G, c, L, seg, gl;
    int i, k;
    bool valid;
    int64_t base;
};

// The next work item at or after `item` whose system takes part in the wave.
// vw: rows per access of the asking instance, which takes systems whose line
// pitch is a multiple of vw only (the one-row instance takes every system).
// padded: the arrays are the mixed form's padded FP32 ones (pitch SysDev::jp).
// kind: which line kernel asks (SysDev::line_kind: warp-staged or one lane per
// line); each takes its own systems.  pf: the system of `item` when the caller
// has already loaded it, else -1.
__device__ __forceinline__ bool next_line_job(const BatchView &b, const WaveArgs &w, int item, int step, int total,
                                              int lane, int vw, bool padded, int kind, LineJob &j, int pf = -1)
{
    for (; item < total; item += step, pf = -1) {
        const int sidx = (w.kind == 0) ? (pf >= 0 ? pf : __ldg(b.line_sys + item)) : 0;
        if (!gate_ok(b.st[sidx], w.gate)) continue;
        const SysDev &d = b.sys[sidx];
        if (d.line_kind != kind) continue;
        const int lp = padded ? d.jp : d.jmax2;
        if (lp % vw) continue;
        j.item = item;
        j.sidx = sidx;
        j.G = d.lane_group;
        j.c = d.rows_per_lane;
        j.L = d.jmax2;
        j.seg = lane / j.G;
        j.gl = lane - j.seg * j.G;
        const int lpw = 32 / j.G;
        const int item0 = (w.kind == 0) ? b.line_prefix[sidx] : 0;
        const int q = (item - item0) * lpw + j.seg;
        if (w.kind == 0) {
            j.valid = wave_line(d, w, q, j.i, j.k);
        } else if (w.kind == 1) {
            const int ilo = max(1, w.par - d.kmax2), ihi = min(d.imax2, w.par - 1);
            j.i = ilo + q;
            j.k = w.par - j.i;
            j.valid = (j.i <= ihi);
        } else {
            j.valid = q < w.nlines;
            const int2 lk = j.valid ? w.list[q] : make_int2(1, 1);
            j.i = lk.x;
            j.k = lk.y;
        }
        j.base = (int64_t)(j.i - 1) * lp + (int64_t)(j.k - 1) * lp * d.imax2;
        return true;
    }
    j.item = -1;
    return false;
}

// Neighbour-line pointers of a job: the wave's neighbour source, or the line's
// own old values where the neighbour index clamps onto the cell itself.
template <typename T>
__device__ __forceinline__ LineCtx<T> line_ctx(const BatchView &b, const WaveArgs &w, const LineJob &j)
{
    const SysDev &d = b.sys[j.sidx];
    const int64_t c1 = pitch<T>(d), c2 = (int64_t)pitch<T>(d) * d.imax2;
    LineCtx<T> x;
    x.a = diag_base<T>(d);
    x.rhs = vec<T>(d, w.rhs);
    x.n = cells<T>(d);
    x.L = j.L;
    x.do_k = d.do_k;
    x.base = j.base;
    const T *nbr = vec<T>(d, w.nbr), *old = vec<T>(d, w.old);
    // the I and K neighbour lines (clamped onto the line itself at the array
    // edge, wrapped along a cyclic axis)
    const int im = inc_m(j.i - 1, d.imax2, d.cyc & 1), ip = inc_p(j.i - 1, d.imax2, d.cyc & 1);
    const int km = inc_m(j.k - 1, d.kmax2, d.cyc & 4), kp = inc_p(j.k - 1, d.kmax2, d.cyc & 4);
    x.nb_im = im ? nbr + x.base + im * c1 : old + x.base;
    x.nb_ip = ip ? nbr + x.base + ip * c1 : old + x.base;
    x.nb_km = km ? nbr + x.base + km * c2 : old + x.base;
    x.nb_kp = kp ? nbr + x.base + kp * c2 : old + x.base;
    return x;
}

// Right-hand side of row r (operand order of LEQ_IKSWEEP / LEQ_ISWEEP).
template <typename T>
__device__ __forceinline__ T line_rhs(const LineCtx<T> &x, int r)
{
    const int64_t p = x.base + r;
    const int64_t n = x.n;
    T v = x.rhs[p] - x.a[2 * n + p] * x.nb_im[r];
    v = v - x.a[4 * n + p] * x.nb_ip[r];
    if (x.do_k) {
        v = v - x.a[0 * n + p] * x.nb_km[r];
        v = v - x.a[6 * n + p] * x.nb_kp[r];
    }
    return v;
}

// ------------------------------------------------------------------ J-line factorization (once per solve)
// DGTSV's elimination on each J-line's tridiagonal (sub A(-2), diagonal A(0),
// super A(2), CC(first) = EE(last) = 0), run once per solve because the line
// matrices do not change between sweeps.  For a line on which DGTSV takes no
// row interchange and meets no zero pivot the elimination is the LU
// factorization T = L U, stored per row as
//   l_r = a_r / u_{r-1}  (DGTSV's FACT),  r_r = 1 / u_r,  q_r = c_r / u_r,
// so that each sweep only runs the two linear recurrences
//   y_r = f_r - l_r y_{r-1},   x_r = r_r y_r - q_r x_{r+1}.
// The pivot test and the zero-pivot test are DGTSV's own (model/DGTSV.f:109-121,
// 138-163), evaluated on the same values without fused multiply-adds; a line that
// fails them is flagged and solved every sweep by the exact pivoting recurrence.
template <typename T>
__global__ void k_line_factor(BatchView b, const int *all_line_prefix)
{
    const int total = all_line_prefix[b.nsys];
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
        const int s = find_sys(all_line_prefix, b.nsys, g);
        if (!gate_ok(b.st[s], G_INIT)) continue;
        const SysDev &d = b.sys[s];
        const int li = g - all_line_prefix[s];  // (i-1) + (k-1)*imax2
        const int64_t base = (int64_t)li * d.jmax2;       // the line in the FP64 diagonals
        const int64_t fbase = (int64_t)li * pitch<T>(d);  // and in the factor arrays
        const int64_t n = d.n;
        const int L = d.jmax2;
        const double *A = d.a64;
        T *fl = reinterpret_cast<T *>(d.fac[0]) + fbase;
        T *fr = reinterpret_cast<T *>(d.fac[1]) + fbase;
        T *fq = reinterpret_cast<T *>(d.fac[2]) + fbase;
        for (int r = L; r < pitch<T>(d); ++r) fl[r] = fr[r] = fq[r] = T(0);  // pad rows
        int flag = 0;
        double u = A[3 * n + base];
        fl[0] = T(0);
        for (int r = 0; r < L - 1; ++r) {
            const double an = A[1 * n + base + r + 1];  // DL(r)
            const double cr = A[5 * n + base + r];      // DU(r)
            if (!(fabs(u) >= fabs(an)) || u == 0.0) {
                flag = 1;
                break;
            }
            const double l = __ddiv_rn(an, u);
            fr[r] = (T)__ddiv_rn(1.0, u);
            fq[r] = (T)__ddiv_rn(cr, u);
            fl[r + 1] = (T)l;
            u = __dsub_rn(A[3 * n + base + r + 1], __dmul_rn(l, cr));
        }
        if (!flag && u == 0.0) flag = 1;
        if (!flag) {
            fr[L - 1] = (T)__ddiv_rn(1.0, u);
            fq[L - 1] = T(0);
        }
        d.line_flag[li] = flag;
    }
}

// Asynchronous global -> shared copy of B bytes (4, 8 or 16); src_bytes = 0
// fills the destination with zeros and reads nothing.
template <int B>
__device__ __forceinline__ void cp_async(void *smem_dst, const void *gmem_src, int src_bytes)
{
    const unsigned dst = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(dst), "l"(gmem_src), "n"(B), "r"(src_bytes)
                 : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// ------------------------------------------------------------------ J-line half-sweep
// One warp handles 32/G lines, G lanes per line; lane g owns the c rows
// g*c .. g*c+c-1.  Each recurrence is split in three: a pass over the lane's rows
// from a zero start, which yields the chunk's affine map (value at its end as a
// function of the value entering it), a warp scan that composes the maps, and a
// second pass from the entering value.  No division remains in the sweep.
// VW rows per access: a lane reads VW consecutive rows of each operand with one
// load (16 bytes for VW = 4 in FP32 and VW = 2 in FP64), which needs lines that
// start on VW-row boundaries (the mixed form's padded FP32 arrays, pitch a
// multiple of four; an even JMAX2 for two rows).
template <typename T, int VW>
struct alignas(VW * sizeof(T)) RowsV {
    T v[VW];
};
template <typename T, int VW>
__device__ __forceinline__ RowsV<T, VW> ldv(const T *p)
{
    return *reinterpret_cast<const RowsV<T, VW> *>(p);
}

// c - a*b, a*b + c and a*b for the J-line sweeps: in FP32 with every rounding
// stated (so that the register-staged and the bulk-staged kernels give the same
// bits), in FP64 as written.
template <typename T>
__device__ __forceinline__ T fnms(T a, T b, T c) { return c - a * b; }
template <>
__device__ __forceinline__ float fnms<float>(float a, float b, float c) { return __fmaf_rn(-a, b, c); }
template <typename T>
__device__ __forceinline__ T fma_t(T a, T b, T c) { return a * b + c; }
template <>
__device__ __forceinline__ float fma_t<float>(float a, float b, float c) { return __fmaf_rn(a, b, c); }
template <typename T>
__device__ __forceinline__ T mul_t(T a, T b) { return a * b; }
template <>
__device__ __forceinline__ float mul_t<float>(float a, float b) { return __fmul_rn(a, b); }

// The two recurrences of a factored line, y_r = f_r - l_r y_{r-1} and
// x_r = r_r y_r - q_r x_{r+1}, on shared-memory rows: lane gl of the line's G
// lanes owns rows [gl*c, gl*c + c); a pass over the chunk from a zero start gives
// its affine map, a log2(G)-step shuffle scan composes the maps, a second pass
// starts from the entering value.  x replaces f.
template <typename T>
__device__ __forceinline__ void line_recurrences(T *f, const T *fl, const T *fr, const T *fq, int c, int G, int gl)
{
    T *cf = f + gl * c;
    const T *cl = fl + gl * c, *cr = fr + gl * c, *cq = fq + gl * c;
    T mb = T(0), ma = T(1);
#pragma unroll 4
    for (int t = 0; t < c; ++t) {
        const T lt = cl[t];
        mb = fnms(lt, mb, cf[t]);
        ma = -lt * ma;
    }
    for (int dl = 1; dl < G; dl <<= 1) {
        const T pa = __shfl_up_sync(0xffffffffu, ma, dl, G), pb = __shfl_up_sync(0xffffffffu, mb, dl, G);
        if (gl >= dl) {
            mb = fma_t(ma, pb, mb);
            ma = mul_t(ma, pa);
        }
    }
    T y = __shfl_up_sync(0xffffffffu, mb, 1, G);
    if (gl == 0) y = T(0);
#pragma unroll 4
    for (int t = 0; t < c; ++t) {
        y = fnms(cl[t], y, cf[t]);
        cf[t] = y;
    }
    mb = T(0);
    ma = T(1);
#pragma unroll 4
    for (int t = c - 1; t >= 0; --t) {
        const T qt = cq[t];
        mb = fnms(qt, mb, mul_t(cr[t], cf[t]));
        ma = -qt * ma;
    }
    for (int dl = 1; dl < G; dl <<= 1) {
        const T na = __shfl_down_sync(0xffffffffu, ma, dl, G), nb = __shfl_down_sync(0xffffffffu, mb, dl, G);
        if (gl + dl < G) {
            mb = fma_t(ma, nb, mb);
            ma = mul_t(ma, na);
        }
    }
    T xv = __shfl_down_sync(0xffffffffu, mb, 1, G);
    if (gl == G - 1) xv = T(0);
#pragma unroll 4
    for (int t = c - 1; t >= 0; --t) {
        xv = fnms(cq[t], xv, mul_t(cr[t], cf[t]));
        cf[t] = xv;
    }
}

template <typename T, int VW>
__global__ void __launch_bounds__(128, sizeof(T) == 4 ? (VW == 4 ? 5 : 6) : 4) k_jline(BatchView b, WaveArgs w, int cmax)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nwarps = blockDim.x >> 5;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int rows_w = 32 * cmax;
    T *s_f = reinterpret_cast<T *>(smem_raw) + (size_t)warp * 4 * rows_w;
    T *s_l = s_f + rows_w, *s_r = s_l + rows_w, *s_q = s_r + rows_w;

    const int total = (w.kind == 0) ? b.line_prefix[b.nsys] : w.count;
    const int step = gridDim.x * nwarps;
    LineJob j;
    int pf = -1;
    for (int item = blockIdx.x * nwarps + warp; next_line_job(b, w, item, step, total, lane, VW, sizeof(T) == 4, LK_WARP, j, pf);
         item = j.item + step) {
        // the next item's system, loaded while this one is processed
        pf = (w.kind == 0 && j.item + step < total) ? __ldg(b.line_sys + j.item + step) : -1;
        const SysDev &d = b.sys[j.sidx];
        SysState &st = b.st[j.sidx];
        const LineCtx<T> x = line_ctx<T>(b, w, j);
        const int G = j.G, c = j.c, L = j.L, seg = j.seg, gl = j.gl;
        const int segoff = seg * G * c;
        T *f = s_f + segoff, *fl = s_l + segoff, *fr = s_r + segoff, *fq = s_q + segoff;
        const bool exact = j.valid && d.line_flag[(j.i - 1) + (j.k - 1) * d.imax2] != 0;
        const bool fast = j.valid && !exact;
        const T *gl_ = reinterpret_cast<const T *>(d.fac[0]) + x.base;
        const T *gr_ = reinterpret_cast<const T *>(d.fac[1]) + x.base;
        const T *gq_ = reinterpret_cast<const T *>(d.fac[2]) + x.base;


        // ---- load (coalesced over the line): right-hand side and factors.  With an
        // even JMAX2 every line starts on an even cell, so lanes read two rows per
        // access; otherwise U single rows at a time.  The loads do not wait for the
        // line's pivot flag (a flagged line ignores them).
        if constexpr (VW > 1) {  // lines start on VW-row boundaries
            using V = RowsV<T, VW>;
            const int span = G * c;  // a multiple of VW (G >= VW)
            const T *rhs_l = x.rhs + x.base, *am1_l = x.a + 2 * x.n + x.base, *ap1_l = x.a + 4 * x.n + x.base;
            const T *am3_l = x.a + x.base, *ap3_l = x.a + 6 * x.n + x.base;
            for (int r = VW * gl; r < span; r += VW * G) {
                // factors straight to shared memory; rows past the line read the
                // zeros of the pad cells or are zero-filled by the copy
                const bool ok = j.valid && r < L;
                const void *z = d.fac[0];
                cp_async<VW * sizeof(T)>(fl + r, ok ? (const void *)(gl_ + r) : z, ok ? VW * sizeof(T) : 0);
                cp_async<VW * sizeof(T)>(fr + r, ok ? (const void *)(gr_ + r) : z, ok ? VW * sizeof(T) : 0);
                cp_async<VW * sizeof(T)>(fq + r, ok ? (const void *)(gq_ + r) : z, ok ? VW * sizeof(T) : 0);
                V rhs, am1, ap1, am3, ap3, nim, nip, nkm, nkp;
                if (ok) {  // rows r .. r+VW-1 lie on the line or on its pad cells
                    rhs = ldv<T, VW>(rhs_l + r);
                    am1 = ldv<T, VW>(am1_l + r);
                    ap1 = ldv<T, VW>(ap1_l + r);
                    nim = ldv<T, VW>(x.nb_im + r);
                    nip = ldv<T, VW>(x.nb_ip + r);
                    if (x.do_k) {
                        am3 = ldv<T, VW>(am3_l + r);
                        ap3 = ldv<T, VW>(ap3_l + r);
                        nkm = ldv<T, VW>(x.nb_km + r);
                        nkp = ldv<T, VW>(x.nb_kp + r);
                    }
                }
                V fv;
#pragma unroll
                for (int k = 0; k < VW; ++k) {
                    T f0 = T(0);
                    if (fast && r + k < L) {
                        f0 = fnms(am1.v[k], nim.v[k], rhs.v[k]);
                        f0 = fnms(ap1.v[k], nip.v[k], f0);
                        if (x.do_k) {
                            f0 = fnms(am3.v[k], nkm.v[k], f0);
                            f0 = fnms(ap3.v[k], nkp.v[k], f0);
                        }
                    }
                    fv.v[k] = f0;
                }
                *reinterpret_cast<V *>(f + r) = fv;
            }
        } else {
            constexpr int U = 2;
            const T *rhs_l = x.rhs + x.base, *am1_l = x.a + 2 * x.n + x.base, *ap1_l = x.a + 4 * x.n + x.base;
            const T *am3_l = x.a + x.base, *ap3_l = x.a + 6 * x.n + x.base;
            for (int r0 = gl; r0 < G * c; r0 += U * G) {
                T rhs[U], am1[U], ap1[U], am3[U], ap3[U], nim[U], nip[U], nkm[U], nkp[U], lv[U], rv[U], qv[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int r = r0 + u * G;
                    if (j.valid && r < L) {
                        rhs[u] = rhs_l[r];
                        am1[u] = am1_l[r];
                        ap1[u] = ap1_l[r];
                        nim[u] = x.nb_im[r];
                        nip[u] = x.nb_ip[r];
                        if (x.do_k) {
                            am3[u] = am3_l[r];
                            ap3[u] = ap3_l[r];
                            nkm[u] = x.nb_km[r];
                            nkp[u] = x.nb_kp[r];
                        }
                        lv[u] = gl_[r];
                        rv[u] = gr_[r];
                        qv[u] = gq_[r];
                    }
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int r = r0 + u * G;
                    if (r < G * c) {
                        T fv = T(0), l_ = T(0), r_ = T(0), q_ = T(0);
                        if (fast && r < L) {
                            fv = fnms(am1[u], nim[u], rhs[u]);
                            fv = fnms(ap1[u], nip[u], fv);
                            if (x.do_k) {
                                fv = fnms(am3[u], nkm[u], fv);
                                fv = fnms(ap3[u], nkp[u], fv);
                            }
                            l_ = lv[u];
                            r_ = rv[u];
                            q_ = qv[u];
                        }
                        f[r] = fv;
                        fl[r] = l_;
                        fr[r] = r_;
                        fq[r] = q_;
                    }
                }
            }
        }
        if constexpr (VW > 1) cp_async_wait_all();
        __syncwarp();

        line_recurrences<T>(f, fl, fr, fq, c, G, gl);
        __syncwarp();

        // ---- lines on which DGTSV interchanges rows or meets a zero pivot
        const unsigned segmask = (G == 32 ? 0xffffffffu : ((1u << G) - 1u)) << (seg * G);
        int skip = 0;
        if (exact) {
            for (int r = gl; r < L; r += G) {
                T a_, d_, c_, f_;
                line_row<T>(x, r, a_, d_, c_, f_);
                fl[r] = a_;
                fr[r] = d_;
                fq[r] = c_;
                f[r] = f_;
            }
            __syncwarp(segmask);
            if (gl == 0) {
                skip = dgtsv_rows<T>(L, fl, fr, fq, f) != 0;
                atomicAdd(&st.line_fallbacks, 1);
                if (skip) atomicAdd(&st.line_skips, 1);
            }
            __syncwarp(segmask);
        }
        skip = __shfl_sync(0xffffffffu, skip, seg * G);
        __syncwarp();

        // ---- store: coalesced.  A line left unchanged (INFO != 0) keeps its old value.
        if (j.valid) {
            T *dstp = vec<T>(d, w.dst) + x.base;
            const T *oldl = vec<T>(d, w.old) + x.base;
            if (!skip && VW > 1) {  // VW rows per store; rows past the line are the zeros of its pad cells
                for (int r = VW * gl; r < L; r += VW * G)
                    *reinterpret_cast<RowsV<T, VW> *>(dstp + r) = *reinterpret_cast<const RowsV<T, VW> *>(f + r);
            } else if (!skip) {
                for (int r = gl; r < L; r += G) dstp[r] = f[r];
            } else if (w.write_old) {
                for (int r = gl; r < L; r += G) dstp[r] = oldl[r];
            }
        }
        __syncwarp();
    }
}

// ------------------------------------------------------------------ J-line half-sweep, one lane per line
// For short lines in large numbers (batches and serving) each lane runs the two
// recurrences down its own line, keeping y in the destination (the line's own
// cells, which no other line of the wave reads); no staging, few instructions
// per row.  A flagged line runs DGTSV with interchanges: its matrix rows in the
// line's factor cells (unused for a flagged line), first without the right-hand
// side to find INFO (a line left unchanged on INFO != 0 keeps its old values),
// then, when INFO = 0, again with the right-hand side in the line's own cells of
// the destination.
template <typename T>
__global__ void __launch_bounds__(128) k_jline_thread(BatchView b, WaveArgs w)
{
    const int nwarps = blockDim.x >> 5;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int total = (w.kind == 0) ? b.line_prefix[b.nsys] : w.count;
    const int step = gridDim.x * nwarps;
    LineJob j;
    for (int item = blockIdx.x * nwarps + warp; next_line_job(b, w, item, step, total, lane, 1, sizeof(T) == 4, LK_THREAD, j);
         item = j.item + step) {
        const SysDev &d = b.sys[j.sidx];
        SysState &st = b.st[j.sidx];
        const LineCtx<T> x = line_ctx<T>(b, w, j);
        const int L = j.L;
        const bool exact = j.valid && d.line_flag[(j.i - 1) + (j.k - 1) * d.imax2] != 0;
        const bool fast = j.valid && !exact;
        const T *gl_ = reinterpret_cast<const T *>(d.fac[0]) + x.base;
        const T *gr_ = reinterpret_cast<const T *>(d.fac[1]) + x.base;
        const T *gq_ = reinterpret_cast<const T *>(d.fac[2]) + x.base;
        // ---- one lane per line (short lines, many of them): each lane runs the two
        // recurrences down its own line, keeping y in the destination (the line's
        // own cells, which no other line of the wave reads).
        if (j.valid) {
            T *dstp = vec<T>(d, w.dst) + x.base;
            const T *rhs_l = x.rhs + x.base, *am1_l = x.a + 2 * x.n + x.base, *ap1_l = x.a + 4 * x.n + x.base;
            const T *am3_l = x.a + x.base, *ap3_l = x.a + 6 * x.n + x.base;
            if (fast) {
                T y = T(0);
#pragma unroll 4
                for (int r = 0; r < L; ++r) {
                    T fv = rhs_l[r] - am1_l[r] * x.nb_im[r];
                    fv = fv - ap1_l[r] * x.nb_ip[r];
                    if (x.do_k) {
                        fv = fv - am3_l[r] * x.nb_km[r];
                        fv = fv - ap3_l[r] * x.nb_kp[r];
                    }
                    y = fv - gl_[r] * y;
                    dstp[r] = y;
                }
                T xv = T(0);
#pragma unroll 4
                for (int r = L - 1; r >= 0; --r) {
                    xv = gr_[r] * dstp[r] - gq_[r] * xv;
                    dstp[r] = xv;
                }
            } else {
                // DGTSV with interchanges: the matrix rows in the line's factor cells
                // (unused for a flagged line); INFO first, from the matrix alone
                T *sub = reinterpret_cast<T *>(d.fac[0]) + x.base;
                T *dg = reinterpret_cast<T *>(d.fac[1]) + x.base;
                T *sup = reinterpret_cast<T *>(d.fac[2]) + x.base;
                T f_unused;
                for (int r = 0; r < L; ++r) line_row<T>(x, r, sub[r], dg[r], sup[r], f_unused);
                const int skip = dgtsv_info<T>(L, sub, dg, sup) != 0;
                atomicAdd(&st.line_fallbacks, 1);
                if (skip) {
                    atomicAdd(&st.line_skips, 1);
                    const T *oldl = vec<T>(d, w.old) + x.base;
                    if (w.write_old)
                        for (int r = 0; r < L; ++r) dstp[r] = oldl[r];
                } else {
                    // the right-hand side of row r goes to the line's own cell r of the
                    // destination; a later row reads only its own cell (a neighbour that
                    // clamps onto itself), so the rows are formed before they are overwritten
                    for (int r = 0; r < L; ++r) line_row<T>(x, r, sub[r], dg[r], sup[r], dstp[r]);
                    dgtsv_rows<T>(L, sub, dg, sup, dstp);
                }
            }
        }
    }
}

// ------------------------------------------------------------------ exact sequential line sweeps
// One thread per line, the pivoting DGTSV over global scratch laid out [row][line]
// so that neighbouring threads touch neighbouring words.
template <typename T>
__global__ void k_seq_lines(BatchView b, SeqLineArgs a)
{
    const int li = blockIdx.x * blockDim.x + threadIdx.x;
    if (li >= a.count) return;
    SysState &st = b.st[0];
    if (!gate_ok(st, a.gate)) return;
    const SysDev &d = b.sys[0];
    const int64_t n = cells<T>(d), c1 = pitch<T>(d), c2 = (int64_t)pitch<T>(d) * d.imax2;
    const T *A = diag_base<T>(d);
    const T *rhs = vec<T>(d, a.rhs);
    T *var = vec<T>(d, a.var);
    const int2 lc = a.lines[li];
    int L;
    int64_t base, step;
    // which diagonals form the tridiagonal and which four go to the right-hand side
    int dsub, dsup, o0, o1, o2, o3;
    if (a.axis == 0) {  // I-line at (j,k), LEQ_JKSWEEP: CC=A(-1), EE=A(1)
        L = d.imax2;
        base = (int64_t)(lc.x - 1) + (int64_t)(lc.y - 1) * c2;
        step = c1;
        dsub = 2; dsup = 4; o0 = 1; o1 = 5; o2 = 0; o3 = 6;
    } else if (a.axis == 1) {  // J-line at (i,k), LEQ_IKSWEEP: CC=A(-2), EE=A(2)
        L = d.jmax2;
        base = (int64_t)(lc.x - 1) * c1 + (int64_t)(lc.y - 1) * c2;
        step = 1;
        dsub = 1; dsup = 5; o0 = 2; o1 = 4; o2 = 0; o3 = 6;
    } else {  // K-line at (i,j), LEQ_IJSWEEP: CC=A(-3), EE=A(3)
        L = d.kmax2;
        base = (int64_t)(lc.x - 1) * c1 + (int64_t)(lc.y - 1);
        step = c2;
        dsub = 0; dsup = 6; o0 = 1; o1 = 5; o2 = 2; o3 = 4;
    }
    // RHS operand order follows the reference routines
    T *sub = reinterpret_cast<T *>(a.scratch), *dg = sub + (size_t)a.lmax * a.count,
      *sup = dg + (size_t)a.lmax * a.count, *f = sup + (size_t)a.lmax * a.count;
#define SCR(arr, r) arr[(size_t)(r)*a.count + li]
    for (int r = 0; r < L; ++r) {
        const int64_t p = base + r * step;
        int ii, jj, kk;
        {
            const CellIdx q = cell_ijk_t<T>(d, (uint32_t)p);
            ii = q.i; jj = q.j; kk = q.k;
        }
        auto nb = [&](int dd) -> T {
            int64_t o = 0;
            switch (dd) {
            case 0: o = inc_m(kk, d.kmax2, d.cyc & 4) * c2; break;
            case 1: o = inc_m(jj, d.jmax2, d.cyc & 2); break;
            case 2: o = inc_m(ii, d.imax2, d.cyc & 1) * c1; break;
            case 4: o = inc_p(ii, d.imax2, d.cyc & 1) * c1; break;
            case 5: o = inc_p(jj, d.jmax2, d.cyc & 2); break;
            case 6: o = inc_p(kk, d.kmax2, d.cyc & 4) * c2; break;
            }
            return var[p + o];
        };
        SCR(sub, r) = (r == 0) ? T(0) : A[dsub * n + p];
        SCR(dg, r) = A[3 * n + p];
        SCR(sup, r) = (r == L - 1) ? T(0) : A[dsup * n + p];
        T v = rhs[p] - A[o0 * n + p] * nb(o0);
        v = v - A[o1 * n + p] * nb(o1);
        if (a.axis != 1 || d.do_k) {
            v = v - A[o2 * n + p] * nb(o2);
            v = v - A[o3 * n + p] * nb(o3);
        }
        SCR(f, r) = v;
    }
    // DGTSV on the strided scratch
    int info = 0;
    for (int i = 0; i < L - 1 && !info; ++i) {
        const T dli = SCR(sub, i + 1);
        if (fabs(SCR(dg, i)) >= fabs(dli)) {
            if (SCR(dg, i) != T(0)) {
                const T fact = dli / SCR(dg, i);
                SCR(dg, i + 1) = SCR(dg, i + 1) - fact * SCR(sup, i);
                SCR(f, i + 1) = SCR(f, i + 1) - fact * SCR(f, i);
            } else {
                info = i + 1;
                break;
            }
            if (i < L - 2) SCR(sub, i + 1) = T(0);
        } else {
            const T fact = SCR(dg, i) / dli;
            SCR(dg, i) = dli;
            const T temp = SCR(dg, i + 1);
            SCR(dg, i + 1) = SCR(sup, i) - fact * temp;
            if (i < L - 2) {
                SCR(sub, i + 1) = SCR(sup, i + 1);
                SCR(sup, i + 1) = -fact * SCR(sub, i + 1);
            }
            SCR(sup, i) = temp;
            const T tb = SCR(f, i);
            SCR(f, i) = SCR(f, i + 1);
            SCR(f, i + 1) = tb - fact * SCR(f, i + 1);
        }
    }
    if (!info && SCR(dg, L - 1) == T(0)) info = L;
    if (info) {
        if (a.fatal_on_info)
            atomicOr(&st.err, 2);
        else
            atomicAdd(&st.line_skips, 1);
        return;
    }
    SCR(f, L - 1) = SCR(f, L - 1) / SCR(dg, L - 1);
    if (L > 1) SCR(f, L - 2) = (SCR(f, L - 2) - SCR(sup, L - 2) * SCR(f, L - 1)) / SCR(dg, L - 2);
    for (int i = L - 3; i >= 0; --i)
        SCR(f, i) = (SCR(f, i) - SCR(sup, i) * SCR(f, i + 1) - SCR(sub, i + 1) * SCR(f, i + 2)) / SCR(dg, i);
    for (int r = 0; r < L; ++r) var[base + r * step] = SCR(f, r);
#undef SCR
}

// ------------------------------------------------------------------ standalone kernels
template <typename T>
__global__ void k_matvec_plain(const SysDev *sysp, const T *a, const T *x, T *y)
{
    const SysDev &d = *sysp;
    const int64_t n = d.n;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        const CellIdx q = cell_ijk(d, (uint32_t)c);
        y[c] = (T)stencil_row<T, T>(d, a, x, (uint32_t)c, q);
    }
}

// (x, y) over n values: per-block sums in fixed order, the last block adds them.
__global__ void k_dot(const double *x, const double *y, int64_t n, double *partials, unsigned int *counter,
                      double *out)
{
    __shared__ int last;
    double v[1] = {0.0};
    const int64_t per = (n + gridDim.x - 1) / gridDim.x;
    const int64_t c0 = (int64_t)blockIdx.x * per, c1 = min(n, c0 + per);
    #pragma unroll 4
    for (int64_t c = c0 + threadIdx.x; c < c1; c += blockDim.x) v[0] += x[c] * y[c];
    block_sum<1>(v);
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = v[0];
        __threadfence();
        last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double acc[1] = {0.0};
    for (int t = threadIdx.x; t < (int)gridDim.x; t += blockDim.x) acc[0] += __ldcg(partials + t);
    block_sum<1>(acc);
    if (threadIdx.x == 0) {
        *out = acc[0];
        *counter = 0u;
    }
}

// ------------------------------------------------------------------ LEQ_CG0 (METHOD 5)
// Preconditioned conjugate gradients, FP64 (model/leq_cg.f:96-455).  One
// iteration is Z = MSOLVE(R) (the J-line machinery), then four kernels:
// rho = (R, Z); P = Z + beta P; Q = A P with (P, Q); R -= alpha Q, X += alpha P
// with (R, R).

// Unit scaling by the reciprocal of each row's diagonal, no zero test (:197-211).
__global__ void k_scale_diag(BatchView b)
{
    for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
        const Tile tl = b.tiles[t];
        const SysDev &d = b.sys[tl.sys];
        if (!gate_ok(b.st[tl.sys], G_SETUP)) continue;
        const int64_t n = d.n;
        const int64_t c0 = (int64_t)tl.idx * TILE_CELLS, c1 = min(n, c0 + TILE_CELLS);
        #pragma unroll 4
        for (int64_t c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
            const double oam = 1.0 / d.a64[3 * n + c];
#pragma unroll
            for (int q = 0; q < 7; ++q) d.a64[q * n + c] = d.a64[q * n + c] * oam;
            d.b64[c] = d.b64[c] * oam;
        }
    }
}

// rho(i-1) = (R, Z), its zero test and beta(i-1) (:276-325).
__global__ void __launch_bounds__(256) k_cg_rho(BatchView b, int z_id)
{
    TileRun run{-1, 0};
    auto fin = [&](SysState &st, const double(&tot)[1]) {
        const double rho = tot[0];
        if (rho == 0.0) {  // :294-303, no ITER_TOT update
            st.ier = (st.i != 1) ? -2 : 0;
            st.exit_kind = EX_RHO0;
            st.status = ST_DONE;
            return;
        }
        st.beta = (st.i == 1) ? 0.0 : rho / st.rho;
        st.rho = rho;
    };
    for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
        const Tile tl = b.tiles[t];
        const SysDev &d = b.sys[tl.sys];
        if (!gate_ok(b.st[tl.sys], G_INNER)) continue;
        const int64_t c0 = (int64_t)tl.idx * TILE_CELLS;
        const int cnt = (int)min((int64_t)TILE_CELLS, d.n - c0);
        const double *__restrict__ r = vec<double>(d, V_R) + c0;
        const double *__restrict__ z = vec<double>(d, z_id) + c0;
        double v[1] = {0.0};
        const int np = cnt >> 1;
        for (int q = threadIdx.x; q < np; q += blockDim.x) {
            const double2 rv = ld2(r + 2 * q), zv = ld2(z + 2 * q);
            v[0] += rv.x * zv.x;
            v[0] += rv.y * zv.y;
        }
        if ((cnt & 1) && threadIdx.x == 0) v[0] += r[cnt - 1] * z[cnt - 1];
        tile_partial<1>(b, d, tl.idx, v);
        run_add<1>(b, run, tl.sys, fin);
    }
    run_close<1>(b, run, fin);
}

// P = Z (i = 1) or P = Z + beta P (:305-334).
__global__ void __launch_bounds__(256) k_cg_p(BatchView b, int z_id)
{
    for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
        const Tile tl = b.tiles[t];
        const SysDev &d = b.sys[tl.sys];
        const SysState &st = b.st[tl.sys];
        if (!gate_ok(st, G_INNER)) continue;
        const int64_t c0 = (int64_t)tl.idx * TILE_CELLS;
        const int cnt = (int)min((int64_t)TILE_CELLS, d.n - c0);
        const double *__restrict__ z = vec<double>(d, z_id) + c0;
        double *__restrict__ p = vec<double>(d, V_P) + c0;
        const bool first = st.i == 1;
        const double beta = st.beta;
        const int np = cnt >> 1;
        for (int q = threadIdx.x; q < np; q += blockDim.x) {
            const double2 zv = ld2(z + 2 * q);
            if (first) {
                st2(p + 2 * q, zv);
            } else {
                const double2 pv = ld2(p + 2 * q);
                st2(p + 2 * q, mk2<double>(zv.x + beta * pv.x, zv.y + beta * pv.y));
            }
        }
        if ((cnt & 1) && threadIdx.x == 0) p[cnt - 1] = first ? z[cnt - 1] : z[cnt - 1] + beta * p[cnt - 1];
    }
}

// Q = A P and alpha(i) = rho(i-1) / (P, Q) (:336-354).
__global__ void __launch_bounds__(256) k_cg_matvec(BatchView b)
{
    constexpr int U = 2;
    TileRun run{-1, 0};
    auto fin = [&](SysState &st, const double(&tot)[1]) { st.alpha = st.rho / tot[0]; };
    for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
        const Tile tl = b.tiles[t];
        const SysDev &d = b.sys[tl.sys];
        if (!gate_ok(b.st[tl.sys], G_INNER)) continue;
        const int64_t c0 = (int64_t)tl.idx * TILE_CELLS;
        const int cnt = (int)min((int64_t)TILE_CELLS, d.n - c0);
        const double *__restrict__ a = d.a64;
        const double *__restrict__ p = vec<double>(d, V_P);
        double *__restrict__ q = vec<double>(d, V_V);
        double v[1] = {0.0};
        for (int base = threadIdx.x; base < cnt; base += U * blockDim.x) {
            Row7<double> rw[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int c = base + u * blockDim.x;
                if (c < cnt) load_row7<double, double>(d, a, p, c0 + c, rw[u]);
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int c = base + u * blockDim.x;
                if (c < cnt) {
                    const double yv = dot_row7<double>(rw[u], d.do_k);
                    q[c0 + c] = yv;
                    v[0] += rw[u].x[2] * yv;  // x[2] is P at the cell itself
                }
            }
        }
        tile_partial<1>(b, d, tl.idx, v);
        run_add<1>(b, run, tl.sys, fin);
    }
    run_close<1>(b, run, fin);
}

// R = R - alpha Q, Var = Var + alpha P, Rnorm and the convergence test (:356-410).
__global__ void __launch_bounds__(256) k_cg_xr(BatchView b)
{
    TileRun run{-1, 0};
    auto fin = [&](SysState &st, const double(&tot)[1]) {
        st.rnorm = sqrt(tot[0]);
        if (st.rnorm <= st.tol * st.rnorm0) {  // :396-401
            st.iter_tot_add = st.iter + 1;
            st.ier = 0;
            st.exit_kind = EX_RNORM;
            st.status = ST_DONE;
            return;
        }
        st.iter += 1;
        st.i += 1;
        if (st.i > st.itmax) cg_final(st);
    };
    for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
        const Tile tl = b.tiles[t];
        const SysDev &d = b.sys[tl.sys];
        const SysState &st = b.st[tl.sys];
        if (!gate_ok(st, G_INNER)) continue;
        const int64_t c0 = (int64_t)tl.idx * TILE_CELLS;
        const int cnt = (int)min((int64_t)TILE_CELLS, d.n - c0);
        const double alpha = st.alpha;
        double *__restrict__ r = vec<double>(d, V_R) + c0;
        double *__restrict__ x = vec<double>(d, V_X) + c0;
        const double *__restrict__ p = vec<double>(d, V_P) + c0;
        const double *__restrict__ q = vec<double>(d, V_V) + c0;
        double v[1] = {0.0};
        const int np = cnt >> 1;
        for (int k = threadIdx.x; k < np; k += blockDim.x) {
            const double2 rv = ld2(r + 2 * k), qv = ld2(q + 2 * k), xv = ld2(x + 2 * k), pv = ld2(p + 2 * k);
            const double r0 = rv.x - alpha * qv.x, r1 = rv.y - alpha * qv.y;
            st2(r + 2 * k, mk2<double>(r0, r1));
            st2(x + 2 * k, mk2<double>(xv.x + alpha * pv.x, xv.y + alpha * pv.y));
            v[0] += r0 * r0;
            v[0] += r1 * r1;
        }
        if ((cnt & 1) && threadIdx.x == 0) {
            const int c = cnt - 1;
            const double rv = r[c] - alpha * q[c];
            r[c] = rv;
            x[c] = x[c] + alpha * p[c];
            v[0] += rv * rv;
        }
        tile_partial<1>(b, d, tl.idx, v);
        run_add<1>(b, run, tl.sys, fin);
    }
    run_close<1>(b, run, fin);
}

// ------------------------------------------------------------------ LEQ_GMRES0 (METHOD 3)
// FP64 vector steps of model/leq_gmres.f on one system's device arrays; the
// Hessenberg and Givens scalars live on the host.  Sums are per-block partials
// over a fixed grid, added in block order by one block: deterministic.

// W -= h_prev V_prev (when V_prev is given; h_prev read from device memory),
// then the block partial of (W, V_k): one modified Gram-Schmidt step fused with
// the next one's dot (:303-314).  V_k may be W itself (the final norm).
__global__ void __launch_bounds__(256) k_gm_mgs(double *w, const double *vprev, const double *hprev, const double *vk,
                                                int64_t n, double *partials)
{
    const double h = vprev ? *hprev : 0.0;
    double v[1] = {0.0};
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
        double wv = w[p];
        if (vprev) {
            wv = wv - h * vprev[p];
            w[p] = wv;
        }
        v[0] += wv * vk[p];
    }
    block_sum<1>(v);
    if (threadIdx.x == 0) partials[blockIdx.x] = v[0];
}

// out = the partials added in block order (one block).
__global__ void __launch_bounds__(256) k_gm_sum(const double *partials, int np, double *out)
{
    double v[1] = {0.0};
    for (int t = threadIdx.x; t < np; t += blockDim.x) v[0] += partials[t];
    block_sum<1>(v);
    if (threadIdx.x == 0) *out = v[0];
}

// dst = src * s (V(:,1) = R / NORM_R, V(:,I+1) = WW / H(I+1,I): :283-287, :323-327).
__global__ void __launch_bounds__(256) k_gm_scale(const double *src, double s, double *dst, int64_t n)
{
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x)
        dst[p] = src[p] * s;
}

// t = b - t (TEMP = B - A Var, :221-228).
__global__ void __launch_bounds__(256) k_gm_sub(const double *b, double *t, int64_t n)
{
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x)
        t[p] = b[p] - t[p];
}

// Var += sum_k V(:,k) y(k), the sum over the basis taken per cell in order (:417-426).
__global__ void __launch_bounds__(256) k_gm_update(double *x, const double *V, const double *y, int m, int64_t n)
{
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
        double d = 0.0;
        for (int k = 0; k < m; ++k) d = d + V[(size_t)k * n + p] * y[k];
        x[p] = x[p] + d;
    }
}

// max |b| as the bits of a non-negative double (they order like the values).
__global__ void __launch_bounds__(256) k_gm_maxabs(const double *b, int64_t n, unsigned long long *out)
{
    unsigned long long m = 0;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
        const unsigned long long bits = (unsigned long long)__double_as_longlong(fabs(b[p]));
        m = bits > m ? bits : m;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long other = __shfl_xor_sync(0xffffffffu, m, o);
        m = other > m ? other : m;
    }
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// ------------------------------------------------------------------ LEQ_SOR (METHOD 1)
// model/leq_sor.f: each row times 1/A(ijk,0), A(ijk,0) set to one (:75-85).
__global__ void __launch_bounds__(256) k_sor_scale(const SysDev *sysp, double *a, double *b)
{
    const int64_t n = sysp->n;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
        const double oam = 1.0 / a[3 * n + p];
        a[3 * n + p] = 1.0;
#pragma unroll
        for (int q = 0; q < 7; ++q)
            if (q != 3) a[q * n + p] = a[q * n + p] * oam;
        b[p] = b[p] * oam;
    }
}

// VAR_tmp = VAR + OMEGA (B - sum_nb A_nb VAR_nb - VAR) with OMEGA = 1 and the
// neighbour order of :93-110 (3-D: i, j, k pairs; 2-D: j pair, then i pair).
__global__ void __launch_bounds__(256) k_sor_step(const SysDev *sysp, const double *a, const double *b,
                                                  const double *x, double *tmp)
{
    const SysDev &d = *sysp;
    const int64_t n = d.n;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
        const Offs o = cell_offs(d, (uint32_t)p);
        double v;
        if (d.do_k) {
            v = b[p] - a[2 * n + p] * x[p + o.im];
            v = v - a[4 * n + p] * x[p + o.ip];
            v = v - a[1 * n + p] * x[p + o.jm];
            v = v - a[5 * n + p] * x[p + o.jp];
            v = v - a[0 * n + p] * x[p + o.km];
            v = v - a[6 * n + p] * x[p + o.kp];
        } else {
            v = b[p] - a[1 * n + p] * x[p + o.jm];
            v = v - a[5 * n + p] * x[p + o.jp];
            v = v - a[2 * n + p] * x[p + o.im];
            v = v - a[4 * n + p] * x[p + o.ip];
        }
        v = v - x[p];
        tmp[p] = x[p] + 1.0 * v;
    }
}

// ------------------------------------------------------------------ launchers
#define CHECK_LAUNCH() return cudaGetLastError()

cudaError_t launch_sor(const SysDev *sys_dev, double *a, double *b, double *x, double *tmp, int steps, int64_t n,
                       int grid, cudaStream_t s)
{
    k_sor_scale<<<grid, 256, 0, s>>>(sys_dev, a, b);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || steps < 1) return e;
    k_sor_step<<<grid, 256, 0, s>>>(sys_dev, a, b, x, tmp);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    return cudaMemcpyAsync(x, tmp, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, s);
}

cudaError_t launch_gm_mgs(double *w, const double *vprev, const double *hprev, const double *vk, int64_t n,
                          double *partials, int grid, cudaStream_t s)
{
    k_gm_mgs<<<grid, 256, 0, s>>>(w, vprev, hprev, vk, n, partials);
    CHECK_LAUNCH();
}
cudaError_t launch_gm_sum(const double *partials, int np, double *out, cudaStream_t s)
{
    k_gm_sum<<<1, 256, 0, s>>>(partials, np, out);
    CHECK_LAUNCH();
}
cudaError_t launch_gm_scale(const double *src, double f, double *dst, int64_t n, int grid, cudaStream_t s)
{
    k_gm_scale<<<grid, 256, 0, s>>>(src, f, dst, n);
    CHECK_LAUNCH();
}
cudaError_t launch_gm_sub(const double *b, double *t, int64_t n, int grid, cudaStream_t s)
{
    k_gm_sub<<<grid, 256, 0, s>>>(b, t, n);
    CHECK_LAUNCH();
}
cudaError_t launch_gm_update(double *x, const double *V, const double *y, int m, int64_t n, int grid, cudaStream_t s)
{
    k_gm_update<<<grid, 256, 0, s>>>(x, V, y, m, n);
    CHECK_LAUNCH();
}
cudaError_t launch_gm_maxabs(const double *b, int64_t n, unsigned long long *out, int grid, cudaStream_t s)
{
    k_gm_maxabs<<<grid, 256, 0, s>>>(b, n, out);
    CHECK_LAUNCH();
}

cudaError_t launch_scale_diag(const BatchView &b, const LaunchCfg &c)
{
    k_scale_diag<<<c.cell_grid, CELL_THREADS, 0, c.stream>>>(b);
    CHECK_LAUNCH();
}
cudaError_t launch_cg_rho(const BatchView &b, const LaunchCfg &c, int z_id)
{
    k_cg_rho<<<c.g_p, CELL_THREADS, 0, c.stream>>>(b, z_id);
    CHECK_LAUNCH();
}
cudaError_t launch_cg_p(const BatchView &b, const LaunchCfg &c, int z_id)
{
    k_cg_p<<<c.g_p, CELL_THREADS, 0, c.stream>>>(b, z_id);
    CHECK_LAUNCH();
}
cudaError_t launch_cg_matvec(const BatchView &b, const LaunchCfg &c)
{
    k_cg_matvec<<<c.g_mv, CELL_THREADS, 0, c.stream>>>(b);
    CHECK_LAUNCH();
}
cudaError_t launch_cg_xr(const BatchView &b, const LaunchCfg &c)
{
    k_cg_xr<<<c.g_xr, CELL_THREADS, 0, c.stream>>>(b);
    CHECK_LAUNCH();
}

cudaError_t launch_scale(const BatchView &b, const LaunchCfg &c)
{
    k_scale<<<c.cell_grid, CELL_THREADS, 0, c.stream>>>(b);
    CHECK_LAUNCH();
}
cudaError_t launch_after_scale(const BatchView &b, const LaunchCfg &c)
{
    k_after_scale<<<(b.nsys + 127) / 128, 128, 0, c.stream>>>(b);
    CHECK_LAUNCH();
}
cudaError_t launch_init_done(const BatchView &b, const LaunchCfg &c)
{
    k_init_done<<<(b.nsys + 127) / 128, 128, 0, c.stream>>>(b);
    CHECK_LAUNCH();
}
cudaError_t launch_to_f32(const BatchView &b, const LaunchCfg &c)
{
    k_to_f32<<<c.cell_grid, CELL_THREADS, 0, c.stream>>>(b);
    CHECK_LAUNCH();
}
cudaError_t launch_defl_setup(const BatchView &b, const LaunchCfg &c)
{
    k_defl_setup<<<c.cell_grid, CELL_THREADS, 0, c.stream>>>(b);
    CHECK_LAUNCH();
}
template <typename T>
cudaError_t launch_init_residual(const BatchView &b, const LaunchCfg &c)
{
    k_init_residual<T><<<c.stencil_grid, CELL_THREADS, 0, c.stream>>>(b);
    CHECK_LAUNCH();
}
template <typename T>
cudaError_t launch_init_rtilde(const BatchView &b, const LaunchCfg &c, uint64_t seed)
{
    k_init_rtilde<T><<<c.cell_grid, CELL_THREADS, 0, c.stream>>>(b, seed);
    CHECK_LAUNCH();
}
template <typename T, bool MIXED>
cudaError_t launch_p_update(const BatchView &b, const LaunchCfg &c)
{
    k_p_update<T, MIXED><<<c.g_p, CELL_THREADS, 0, c.stream>>>(b);
    CHECK_LAUNCH();
}
// Shared memory of one warp of the J-line kernel: right-hand side and the three factor rows.
int kernel_smem_line_bytes(int cmax, int elem_bytes) { return 4 * 32 * cmax * elem_bytes; }

// Picks the warps per block that fit the staging buffers, sets the shared-memory
// attribute and returns the resident blocks per SM (0 when a line cannot fit).
template <typename T>
int prepare_line_kernel(int cmax, int *warps)
{
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const int per_warp = kernel_smem_line_bytes(cmax, (int)sizeof(T));
    int wpb = std::min(4, optin / std::max(per_warp, 1));
    if (wpb < 1) return 0;
    *warps = wpb;
    const int smem = wpb * per_warp;
    // the limit is a property of the kernel, shared by every engine of the
    // process (some on other threads): it only ever grows
    static std::mutex mu;
    static int granted = 0;
    constexpr int VMAX = sizeof(T) == 4 ? 4 : 2;  // widest instance
    {
        std::lock_guard<std::mutex> lk(mu);
        if (smem > granted) {
            if (cudaFuncSetAttribute(k_jline<T, VMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
                    cudaSuccess ||
                cudaFuncSetAttribute(k_jline<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
                    cudaSuccess ||
                cudaFuncSetAttribute(k_jline<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
                    cudaSuccess)
                return 0;
            granted = smem;
        }
    }
    int nb = 0, nb1 = 0, nb2 = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_jline<T, VMAX>, wpb * 32, smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb2, k_jline<T, 2>, wpb * 32, smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb1, k_jline<T, 1>, wpb * 32, smem) != cudaSuccess)
        return 0;
    return std::min(nb, std::min(nb1, nb2));
}

template <typename T>
int line_thread_occupancy()
{
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_jline_thread<T>, 128, 0) != cudaSuccess) {
        cudaGetLastError();
        return 4;
    }
    return nb > 0 ? nb : 1;
}

// Resident blocks per SM of the staged matvec (shared memory above the default
// limit is requested first); 0 when it cannot run.
template <int CFG>
static int staged_occupancy_cfg()
{
    const int smem = (int)mv_smem<CFG>();
    int nb = 0;
    if (cudaFuncSetAttribute(k_matvec_staged<0, CFG>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) ==
            cudaSuccess &&
        cudaFuncSetAttribute(k_matvec_staged<1, CFG>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) ==
            cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_matvec_staged<1, CFG>, MV_BLOCK, smem) == cudaSuccess) {
        cudaGetLastError();
        return nb;
    }
    cudaGetLastError();
    return 0;
}

// Resident blocks per SM of the staged matvec shape CFG (shared memory above the
// default limit is requested first); 0 when it cannot run.
static int staged_occupancy(int cfg)
{
    switch (cfg) {
    case 1: return staged_occupancy_cfg<1>();
    case 2: return staged_occupancy_cfg<2>();
    default: return 0;
    }
}

template <int KIND>
static void launch_staged(const BatchView &b, const LaunchCfg &c, int src)
{
    switch (c.mv_staged) {
    case 1: k_matvec_staged<KIND, 1><<<c.g_mv_staged, MV_BLOCK, mv_smem<1>(), c.stream>>>(b, src); break;
    default: k_matvec_staged<KIND, 2><<<c.g_mv_staged, MV_BLOCK, mv_smem<2>(), c.stream>>>(b, src); break;
    }
}

template <typename K>
static int occ(K kern)
{
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, CELL_THREADS, 0) != cudaSuccess) {
        cudaGetLastError();
        return 2;
    }
    return nb > 0 ? nb : 1;
}

// Resident blocks per SM of each cell kernel (persistent grids).
void cell_occupancy(bool fp32, CellOcc *o)
{
    if (fp32) {
        o->p_update = occ(k_p_update<float, true>);
        o->s_update = occ(k_s_update<float, true>);
        o->xr_update = occ(k_xr_update<float, true>);
        o->matvec = occ(k_matvec_omega<float, true, false>);
        o->matvec_pair = occ(k_matvec_omega<float, true, true>);
        for (int q = 1; q <= MV_SHAPES; ++q) o->matvec_staged[q] = staged_occupancy(q);
        cudaGetLastError();
        o->copy = occ(k_copy<float>);
        o->outer = occ(k_outer_step);
    } else {
        o->p_update = occ(k_p_update<double, false>);
        o->s_update = occ(k_s_update<double, false>);
        o->xr_update = occ(k_xr_update<double, false>);
        o->matvec = occ(k_matvec_omega<double, false, false>);
        o->matvec_pair = occ(k_matvec_omega<double, false, true>);
        o->copy = occ(k_copy<double>);
        o->outer = occ(k_outer_step);
    }
}

template <typename T>
cudaError_t launch_jline(const BatchView &b, const LaunchCfg &c, const WaveArgs &w)
{
    // systems with one lane per line, then those with several: one warp-kernel
    // launch, the two-row instance when all their lines have even length
    if (c.line_thread) k_jline_thread<T><<<c.line_grid_thread, 128, 0, c.stream>>>(b, w);
    if (c.line_warp) {
        const int smem = c.line_warps * kernel_smem_line_bytes(c.line_cmax, (int)sizeof(T));
        constexpr int VMAX = sizeof(T) == 4 ? 4 : 2;
        if (c.line_single || c.line_vw == 1)
            k_jline<T, 1><<<c.line_grid, c.line_warps * 32, smem, c.stream>>>(b, w, c.line_cmax);
        else if (c.line_vw >= VMAX)
            k_jline<T, VMAX><<<c.line_grid, c.line_warps * 32, smem, c.stream>>>(b, w, c.line_cmax);
        else
            k_jline<T, 2><<<c.line_grid, c.line_warps * 32, smem, c.stream>>>(b, w, c.line_cmax);
    }
    CHECK_LAUNCH();
}
template <typename T>
cudaError_t launch_diag(const BatchView &b, const LaunchCfg &c, int src, int dst, int gate)
{
    k_diag<T><<<c.g_copy, CELL_THREADS, 0, c.stream>>>(b, src, dst, gate);
    CHECK_LAUNCH();
}
template <typename T>
cudaError_t launch_copy(const BatchView &b, const LaunchCfg &c, int src, int dst, int gate)
{
    k_copy<T><<<c.g_copy, CELL_THREADS, 0, c.stream>>>(b, src, dst, gate);
    CHECK_LAUNCH();
}
template <typename T, bool MIXED>
cudaError_t launch_matvec_alpha(const BatchView &b, const LaunchCfg &c, int src)
{
    // the mixed form's padded FP32 arrays: operands staged by bulk copies
    if (MIXED && sizeof(T) == 4 && c.mv_staged) {
        launch_staged<0>(b, c, src);
        CHECK_LAUNCH();
    }
    // two-cell rows for systems with an even JMAX2, one-cell rows for the others
    if (c.rows_pair) k_matvec_alpha<T, MIXED, true><<<c.g_mv_pair, CELL_THREADS, 0, c.stream>>>(b, src);
    if (c.rows_single) k_matvec_alpha<T, MIXED, false><<<c.g_mv, CELL_THREADS, 0, c.stream>>>(b, src);
    CHECK_LAUNCH();
}
template <typename T, bool MIXED>
cudaError_t launch_s_update(const BatchView &b, const LaunchCfg &c)
{
    k_s_update<T, MIXED><<<c.g_s, CELL_THREADS, 0, c.stream>>>(b);
    CHECK_LAUNCH();
}
template <typename T, bool MIXED>
cudaError_t launch_matvec_omega(const BatchView &b, const LaunchCfg &c, int src)
{
    if (MIXED && sizeof(T) == 4 && c.mv_staged) {
        launch_staged<1>(b, c, src);
        CHECK_LAUNCH();
    }
    if (c.rows_pair) k_matvec_omega<T, MIXED, true><<<c.g_mv_pair, CELL_THREADS, 0, c.stream>>>(b, src);
    if (c.rows_single) k_matvec_omega<T, MIXED, false><<<c.g_mv, CELL_THREADS, 0, c.stream>>>(b, src);
    CHECK_LAUNCH();
}
template <typename T, bool MIXED>
cudaError_t launch_xr_update(const BatchView &b, const LaunchCfg &c, int ph, int sh)
{
    k_xr_update<T, MIXED><<<c.g_xr, CELL_THREADS, 0, c.stream>>>(b, ph, sh);
    CHECK_LAUNCH();
}
template <typename T>
cudaError_t launch_line_factor(const BatchView &b, const LaunchCfg &c, const int *all_line_prefix, int total_lines)
{
    if (total_lines <= 0) return cudaSuccess;
    k_line_factor<T><<<(total_lines + 127) / 128, 128, 0, c.stream>>>(b, all_line_prefix);
    CHECK_LAUNCH();
}
// The per-system states written straight into pinned host memory by the SMs
// (posted writes over the host link), not by a copy engine: a state read the host
// polls on never queues behind bulk copies in flight on other streams (the scaled
// A_M / B_M going back during the iterations, serving requests' inputs and results).
static_assert(sizeof(SysState) % 8 == 0, "SysState copied in 8-byte words");
__global__ void __launch_bounds__(256) k_state_snapshot(const SysState *__restrict__ src, SysState *dst, int nsys)
{
    const int64_t words = (int64_t)nsys * (int64_t)(sizeof(SysState) / 8);
    const unsigned long long *s = reinterpret_cast<const unsigned long long *>(src);
    unsigned long long *d = reinterpret_cast<unsigned long long *>(dst);
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < words; q += (int64_t)gridDim.x * blockDim.x)
        d[q] = __ldcg(s + q);
}

cudaError_t launch_state_snapshot(const SysState *src, SysState *dst_host, int nsys, cudaStream_t s)
{
    if (nsys <= 0) return cudaSuccess;
    const int64_t words = (int64_t)nsys * (int64_t)(sizeof(SysState) / 8);
    const int grid = (int)std::min<int64_t>(64, (words + 255) / 256);
    k_state_snapshot<<<grid, 256, 0, s>>>(src, dst_host, nsys);
    return cudaGetLastError();
}

cudaError_t launch_outer_step(const BatchView &b, const LaunchCfg &c)
{
    k_outer_step<<<c.g_outer, CELL_THREADS, 0, c.stream>>>(b);
    CHECK_LAUNCH();
}
template <typename T>
cudaError_t launch_matvec_plain(const SysDev *sys_dev, const SysDev &h, const T *a, const T *x, T *y,
                                cudaStream_t s, int grid)
{
    (void)h;
    k_matvec_plain<T><<<grid, CELL_THREADS, 0, s>>>(sys_dev, a, x, y);
    CHECK_LAUNCH();
}
cudaError_t launch_dot(const double *x, const double *y, int64_t n, double *partials, unsigned int *counter,
                       double *out, int grid, cudaStream_t s)
{
    k_dot<<<grid, CELL_THREADS, 0, s>>>(x, y, n, partials, counter, out);
    CHECK_LAUNCH();
}
template <typename T>
cudaError_t launch_seq_lines(const BatchView &b, const SeqLineArgs &a, cudaStream_t s)
{
    if (a.count <= 0) return cudaSuccess;
    k_seq_lines<T><<<(a.count + 127) / 128, 128, 0, s>>>(b, a);
    CHECK_LAUNCH();
}

// explicit instantiations
#define INST_T(T)                                                                                        \
    template cudaError_t launch_init_residual<T>(const BatchView &, const LaunchCfg &);                  \
    template cudaError_t launch_init_rtilde<T>(const BatchView &, const LaunchCfg &, uint64_t);          \
    template cudaError_t launch_jline<T>(const BatchView &, const LaunchCfg &, const WaveArgs &);        \
    template cudaError_t launch_diag<T>(const BatchView &, const LaunchCfg &, int, int, int);            \
    template cudaError_t launch_copy<T>(const BatchView &, const LaunchCfg &, int, int, int);            \
    template cudaError_t launch_matvec_plain<T>(const SysDev *, const SysDev &, const T *, const T *, T *, \
                                                cudaStream_t, int);                                       \
    template cudaError_t launch_seq_lines<T>(const BatchView &, const SeqLineArgs &, cudaStream_t);        \
    template int prepare_line_kernel<T>(int, int *);                                                     \
    template int line_thread_occupancy<T>();                                                             \
    template cudaError_t launch_line_factor<T>(const BatchView &, const LaunchCfg &, const int *, int);
#define INST_TM(T, M)                                                                       \
    template cudaError_t launch_p_update<T, M>(const BatchView &, const LaunchCfg &);       \
    template cudaError_t launch_matvec_alpha<T, M>(const BatchView &, const LaunchCfg &, int); \
    template cudaError_t launch_s_update<T, M>(const BatchView &, const LaunchCfg &);       \
    template cudaError_t launch_matvec_omega<T, M>(const BatchView &, const LaunchCfg &, int); \
    template cudaError_t launch_xr_update<T, M>(const BatchView &, const LaunchCfg &, int, int);
INST_T(double)
INST_T(float)
INST_TM(double, false)
INST_TM(float, true)

}  // namespace mfixgpu
