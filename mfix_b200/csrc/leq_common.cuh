// leq_common.cuh -- device-side data structures shared by every kernel of the
// B200 linear-equation path (SOLVE_LIN_EQ -> LEQ_BICGS of MFIX 2016-1).
//
// Everything is batch-shaped: a "system" is one A_M(:,:,M) / B_M(:,M) / VAR
// triple on one box geometry, and every kernel walks a device-resident table of
// systems.  The single-system drop-in is a batch of one.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace mfixgpu {

// Work vectors of LEQ_BICGS0 (model/leq_bicgs.f:171-176) plus the solution.
enum VecId : int {
    V_X = 0,  // VAR (unused slot in the mixed form, which accumulates into x64[0])
    V_R,      // R
    V_RT,     // Rtilde
    V_P,      // P
    V_PH,     // P_preconditioned
    V_S,      // Svec
    V_SH,     // Svec_preconditioned
    V_T,      // Tvec
    V_V,      // V
    NVEC
};

enum PcKind : int { PC_NONE = 0, PC_DIAG = 1, PC_LINE = 2 };

enum Status : int { ST_RUNNING = 0, ST_DONE = 1 };
// PH_SETUP: unit scaling pending; PH_INIT: line factors / FP32 copy / initial
// residual pending; then PH_INNER (BiCGSTAB iterations) and, in the mixed form,
// PH_OUTER (FP64 reliable update).
enum Phase : int { PH_INNER = 0, PH_OUTER = 1, PH_SETUP = 2, PH_INIT = 3 };

// exit_kind values reported per solve
enum ExitKind : int {
    EX_RNORM = 0,     // Rnorm <= TOL*Rnorm0 (model/leq_bicgs.f:455-460)
    EX_SNORM = 1,     // Snorm <= TOLMIN (:375-395)
    EX_RHO0 = 2,      // rho == 0 (:320-332)
    EX_ITMAX = 3,     // loop exhausted (:485-495)
    EX_SINGULAR = 4,  // zero row during unit scaling (:217-233)
    EX_ERROR = 5,
    EX_FALLBACK = 6   // mixed form gave up (divergence / stagnation): re-solved in FP64
};

// Magic-number unsigned division by a runtime constant (round-up method,
// Granlund & Montgomery 1994): q = (umulhi(n, m) + n) >> l, valid for n < 2^32.
struct FastDiv {
    uint32_t d, m, l;
};

__host__ __device__ inline FastDiv make_fastdiv(uint32_t d)
{
    FastDiv f;
    f.d = d;
    uint32_t l = 0;
    while ((1ull << l) < d) ++l;
    f.l = l;
    f.m = (uint32_t)(((((uint64_t)1) << 32) * ((((uint64_t)1) << l) - d)) / d + 1);
    return f;
}

__device__ __forceinline__ uint32_t fdiv(uint32_t n, const FastDiv &f)
{
    return (uint32_t)(((uint64_t)__umulhi(n, f.m) + n) >> f.l);
}

// J-line kernels: lanes of one warp share a line and stage its rows through
// registers (k_jline), or one lane runs a whole line (k_jline_thread).
enum LineKind : int { LK_WARP = 0, LK_THREAD = 1 };

// One system of the batch.
struct SysDev {
    int imax2, jmax2, kmax2, do_k;
    int64_t n;           // DIMENSION_3 (cells incl. the wall layer)
    // Layout of the arrays in the form's working precision.  The FP64 drop-in
    // works on the caller's arrays (line pitch JMAX2, n cells).  The mixed form's
    // FP32 arrays (diagonals, factors, vectors) are its own: each J-line padded to
    // a pitch that is a multiple of four cells, so every line starts on a 16-byte
    // boundary; the pad cells hold zeros (diagonal A(0) = 1).
    int cyc;             // cyclic axes (1 I, 2 J, 4 K): the interior cells' neighbours wrap
    int jp;              // line pitch of those arrays
    int64_t np;          // their cells: jp * imax2 * kmax2
    FastDiv div_jp;      // division by jp
    FastDiv div_j;       // division by jmax2
    FastDiv div_i;       // division by imax2
    FastDiv div_h;       // division by half_lines
    int pc;              // PcKind
    int ntiles;          // cell tiles of this system
    int tile_base;       // first tile's slot in the partial-sum array
    int lane_group;      // G: lanes that share one J-line (power of two <= 32)
    int line_kind;       // LineKind: which J-line kernel sweeps this system's lines
    int rows_per_lane;   // c: rows of a line each lane owns (G*c >= jmax2)
    int half_lines;      // ceil(imax2/2): parity-wave slots per k row
    double *a64;         // 7*n diagonals, Fortran A_M(DIMENSION_3,-3:3) order
    double *b64;         // B_M(:,M)
    double *x64[2];      // VAR; x64[1] keeps the initial guess in the mixed form (FP64 re-solve)
    float *a32;          // FP32 copy of the scaled diagonals (mixed form)
    float *defect;       // mixed form: row sums of the scaled A, formed in FP64 (A x = sum a_nb (x_nb - x) + defect x)
    unsigned char *defl_z;  // mixed form: 1 on rows coupled to a neighbour, 0 on decoupled (wall) rows
    float *defl_az;      // mixed form, deflated systems: A z, formed in FP64
    void *vec[NVEC];     // work vectors, double or float by precision
    void *fac[3];        // J-line LU factors per cell (l, 1/u, c/u), double or float by precision
    int *line_flag;      // per J-line (i-1)+(k-1)*imax2: 1 where DGTSV interchanges rows or meets a zero pivot
};

// Per-system solver state, device resident; the scalars of LEQ_BICGS0 plus
// the bookkeeping the reference keeps in locals and ITER_TOT.
struct SysState {
    double rho, rho_prev, alpha, omega, beta;
    double rnorm0, rnorm, snorm;
    double tol;           // TOL
    double outer_rnorm0;  // mixed form: ||b - A x0|| in FP64
    double outer_rnorm;   // mixed form: latest FP64 true residual
    double inner_tol;     // mixed form: residual drop (vs maxr) that triggers a reliable update
    double maxr;          // mixed form: largest recursive residual since the last reliable update
    double best;          // mixed form: smallest true residual seen at a reliable update
    double growth_limit;  // mixed form: hand over when a true residual exceeds growth_limit * best
    double min_margin;    // mixed form: systems whose diagonal-dominance margin is below this go to FP64
    unsigned int margin_bits;  // mixed form: min over rows of |row sum| / |A(0)| (float bits, set in setup)
    int stall_limit;      // mixed form: hand over after this many updates without a 10% gain
    int itmax;
    int i;                // reference loop index of the next iteration (1-based)
    int iter;             // reference ITER counter
    int status;           // Status
    int ier;
    int exit_kind;
    int iter_tot_add;
    int snorm_exit;
    int phase;            // Phase
    int outer_steps;
    int inner_total;      // inner iterations summed over outer steps
    int inner_first;      // mixed form: the correction d restarts from zero at the next X update
    int xcur;             // mixed form: which x64 buffer holds VAR
    int restart;          // mixed form: next reliable update restarts the Krylov process (Rtilde = R)
    int stall;            // mixed form: reliable updates since the best true residual improved by 10%
    int mixed;            // 1: mixed form (setup ends in PH_OUTER), 0: FP64 drop-in
    int method;           // LEQ_METHOD: 2 BiCGSTAB, 5 CG
    int line_skips;       // J-lines left unchanged because DGTSV reported INFO != 0
    int line_fallbacks;   // J-lines solved by the sequential pivoting path
    int defl_allow;       // mixed form: a system below min_margin may be deflated instead of handed over
    int defl;             // mixed form: the inner iteration deflates z (coupled-row indicator)
    double defl_e;        // z^T A z
    double defl_cp, defl_cs;  // z^T P / z^T A z and z^T S / z^T A z of the current iteration
    int replace_every;    // mixed form, deflated systems: FP64 residual replacement at least every this many iterations
    int icheck;           // FP64 BiCGSTAB: 0, or MINIMIZE_DOTPRODUCTS with the Rnorm test every icheck iterations
    double restart_growth;  // mixed form, deflated systems: restart the Krylov process when a true residual exceeds
                            // this multiple of the best (0: never)
    int since_outer;      // mixed form: inner iterations since the last FP64 update
    int err;
    unsigned int arrivals;  // tiles that finished the current reduction kernel
};

// One cell tile: TILE consecutive cells of one system.
struct Tile {
    int sys;
    int idx;  // tile index within the system
};

constexpr int TILE_CELLS = 4096;
constexpr int CELL_THREADS = 256;

// Ordered parameters of one J-line half-sweep (a "wave").
// Along a cyclic axis with an odd number of interior cells the first and last
// interior lines wrap onto each other with the same red/black colour; in the
// reference's loop order (k outer, i inner) the last one comes second and sees the
// first one's new value.  A line's wrap level counts such late positions: a
// colour's lines run level by level.
__host__ __device__ __forceinline__ int wrap_level(const SysDev &d, int i, int k)
{
    int l = 0;
    if ((d.cyc & 1) && ((d.imax2 - 2) & 1) && i == d.imax2 - 1) ++l;
    if (d.do_k && (d.cyc & 4) && ((d.kmax2 - 2) & 1) && k == d.kmax2 - 1) ++l;
    return l;
}

struct WaveArgs {
    int kind;        // 0: lines with ((i + k) & 1) == par, 1: lines with i + k == diag, 2: single line list
    int par;         // parity or diagonal index
    int rhs, nbr, old, dst;  // VecId of the right-hand side, neighbour source, own-old source, output
    int write_old;   // lines skipped on INFO != 0 copy their old value into dst
    int gate;        // which systems take part (see gate_ok)
    int count;       // kinds 1 and 2 (single system): work items in the wave
    int nlines;      // kind 2: lines in `list`
    const int2 *list;  // kind 2: (i, k) of each line, 1-based
    int lvl;         // kind 0: 0 every line of the parity, else only lines of wrap level lvl - 1
};

enum Gate : int {
    G_INNER = 0,        // running, inner phase
    G_INNER_NOSNORM = 1,// running, inner phase, no Snorm exit this iteration
    G_OUTER = 2,        // running, outer phase
    G_ANY = 3,          // running
    G_SETUP = 4,        // running, scaling pending
    G_INIT = 5          // running, setup after scaling pending
};

__device__ __forceinline__ bool gate_ok(const SysState &s, int gate)
{
    if (s.status != ST_RUNNING) return false;
    switch (gate) {
    case G_INNER: return s.phase == PH_INNER;
    case G_INNER_NOSNORM: return s.phase == PH_INNER && !s.snorm_exit;
    case G_OUTER: return s.phase == PH_OUTER;
    case G_SETUP: return s.phase == PH_SETUP;
    case G_INIT: return s.phase == PH_INIT;
    default: return true;
    }
}

}  // namespace mfixgpu
