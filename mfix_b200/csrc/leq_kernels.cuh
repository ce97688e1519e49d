// leq_kernels.cuh -- launch interface of the B200 kernels for the LEQ_BICGS path.
#pragma once
#include "leq_common.cuh"

namespace mfixgpu {

// Everything a kernel needs to find the batch.
struct BatchView {
    const SysDev *sys;     // [nsys]
    SysState *st;          // [nsys]
    const Tile *tiles;     // [ntiles]
    int ntiles;
    int nsys;
    const int *line_prefix;  // [nsys+1] parity-wave work items (exclusive prefix)
    const int *line_sys;     // [items] the system of each parity-wave work item
    double *partials;        // [ntiles_total * 2]
};

struct LaunchCfg {
    int cell_grid;     // blocks of the setup cell kernels (one per tile)
    int stencil_grid;  // blocks of the setup stencil kernels
    int g_p, g_s, g_xr, g_mv, g_copy, g_outer;  // persistent grids of the iteration kernels
    int g_mv_pair;        // grid of the matvec kernels' two-cell form
    int rows_pair;        // 1: some system has an even JMAX2 (two-cell matvec rows)
    int rows_single;      // 1: some system has an odd JMAX2 (one-cell matvec rows)
    int mv_staged;        // mixed form: the matvecs stage their operands by bulk copies (1), without x's
                          // line / plane windows (2), or load them per thread (0)
    int g_mv_staged;      // grid of the staged matvec
    int line_grid;   // blocks for J-line kernels
    int line_cmax;   // max rows per lane over the batch (smem sizing)
    int line_warps;  // warps per block of the J-line kernel
    int line_grid_thread;  // blocks of the one-lane-per-line kernel (4 warps each)
    int line_thread;       // 1: some system has one lane per line
    int line_warp;         // 1: some system has several lanes per line
    int line_single;       // 1: some system with several lanes per line has an odd line pitch
    int line_vw;           // rows per access of the warp J-line kernel (1, 2 or 4)
    cudaStream_t stream;
};

// Setup
cudaError_t launch_scale(const BatchView &b, const LaunchCfg &c);
cudaError_t launch_after_scale(const BatchView &b, const LaunchCfg &c);
cudaError_t launch_to_f32(const BatchView &b, const LaunchCfg &c);
cudaError_t launch_defl_setup(const BatchView &b, const LaunchCfg &c);  // mixed form: A z and z^T A z
cudaError_t launch_init_done(const BatchView &b, const LaunchCfg &c);
cudaError_t launch_scale_diag(const BatchView &b, const LaunchCfg &c);  // LEQ_CG0's scaling by A(0)
template <typename T>
cudaError_t launch_init_residual(const BatchView &b, const LaunchCfg &c);  // R = B - A X, ||R||
template <typename T>
cudaError_t launch_init_rtilde(const BatchView &b, const LaunchCfg &c, uint64_t seed);  // Rtilde, rho(0)

// One CG iteration after Z = MSOLVE(R) (model/leq_cg.f:271-410), FP64
cudaError_t launch_cg_rho(const BatchView &b, const LaunchCfg &c, int z_id);  // rho = (R, Z), beta
cudaError_t launch_cg_p(const BatchView &b, const LaunchCfg &c, int z_id);    // P = Z + beta P
cudaError_t launch_cg_matvec(const BatchView &b, const LaunchCfg &c);         // Q = A P, alpha
cudaError_t launch_cg_xr(const BatchView &b, const LaunchCfg &c);             // R, Var, Rnorm, exit

// LEQ_SOR (model/leq_sor.f): the scaling, then (steps >= 1) one point-Jacobi step through tmp
cudaError_t launch_sor(const SysDev *sys_dev, double *a, double *b, double *x, double *tmp, int steps, int64_t n,
                       int grid, cudaStream_t s);

// LEQ_GMRES0 vector steps (model/leq_gmres.f), FP64 on raw device arrays
cudaError_t launch_gm_mgs(double *w, const double *vprev, const double *hprev, const double *vk, int64_t n,
                          double *partials, int grid, cudaStream_t s);  // W -= h V_prev; partials of (W, V_k)
cudaError_t launch_gm_sum(const double *partials, int np, double *out, cudaStream_t s);
cudaError_t launch_gm_scale(const double *src, double f, double *dst, int64_t n, int grid, cudaStream_t s);
cudaError_t launch_gm_sub(const double *b, double *t, int64_t n, int grid, cudaStream_t s);  // t = b - t
cudaError_t launch_gm_update(double *x, const double *V, const double *y, int m, int64_t n, int grid,
                             cudaStream_t s);  // x += V y
cudaError_t launch_gm_maxabs(const double *b, int64_t n, unsigned long long *out, int grid, cudaStream_t s);

// J-line LU factors (l, 1/u, c/u) and DGTSV pivot flags, once per solve
template <typename T>
cudaError_t launch_line_factor(const BatchView &b, const LaunchCfg &c, const int *all_line_prefix, int total_lines);

// One BiCGSTAB iteration (model/leq_bicgs.f:316-466)
template <typename T, bool MIXED>
cudaError_t launch_p_update(const BatchView &b, const LaunchCfg &c);
template <typename T>
cudaError_t launch_jline(const BatchView &b, const LaunchCfg &c, const WaveArgs &w);
template <typename T>
cudaError_t launch_diag(const BatchView &b, const LaunchCfg &c, int src, int dst, int gate);
template <typename T>
cudaError_t launch_copy(const BatchView &b, const LaunchCfg &c, int src, int dst, int gate);
template <typename T, bool MIXED>
cudaError_t launch_matvec_alpha(const BatchView &b, const LaunchCfg &c, int src);   // V = A*Phat, alpha
template <typename T, bool MIXED>
cudaError_t launch_s_update(const BatchView &b, const LaunchCfg &c);               // S = R - alpha V, Snorm
template <typename T, bool MIXED>
cudaError_t launch_matvec_omega(const BatchView &b, const LaunchCfg &c, int src);   // T = A*Shat, omega
template <typename T, bool MIXED>
cudaError_t launch_xr_update(const BatchView &b, const LaunchCfg &c, int ph, int sh);  // X, R, Rnorm, rho

// Mixed form: FP64 refinement step (outer residual in FP64, x accumulated in FP64)
cudaError_t launch_outer_step(const BatchView &b, const LaunchCfg &c);
// The states of nsys systems copied by the SMs into pinned (device-accessible) host memory.
cudaError_t launch_state_snapshot(const SysState *src, SysState *dst_host, int nsys, cudaStream_t s);

// Standalone kernels behind the per-routine C entry points
template <typename T>
cudaError_t launch_matvec_plain(const SysDev *sys_dev, const SysDev &h, const T *a, const T *x, T *y,
                                cudaStream_t s, int grid);
cudaError_t launch_dot(const double *x, const double *y, int64_t n, double *partials, unsigned int *counter,
                       double *out, int grid, cudaStream_t s);
// Sequential-per-thread exact DGTSV over a list of lines along I or K (LEQ_JKSWEEP / LEQ_IJSWEEP)
// or J (lexicographic / ASAS IK order), writing the error flag on INFO != 0 where the reference aborts.
struct SeqLineArgs {
    int axis;           // 0: line along I at (j,k); 1: along J at (i,k); 2: along K at (i,j)
    const int2 *lines;  // line coordinates (1-based)
    int count;
    int rhs, var;       // VecId of right-hand side and of the vector being swept in place
    int fatal_on_info;  // 1: INFO != 0 is an error (JK / IJ sweeps), 0: skip the line (IK sweep)
    double *scratch;    // 4 * Lmax * count values
    int lmax;
    int gate;           // which systems take part (Gate)
};
template <typename T>
cudaError_t launch_seq_lines(const BatchView &b, const SeqLineArgs &a, cudaStream_t s);

int kernel_smem_line_bytes(int cmax, int elem_bytes);
template <typename T>
int prepare_line_kernel(int cmax, int *warps);
template <typename T>
int line_thread_occupancy();  // resident blocks per SM of the one-lane-per-line kernel
//  // sets the smem attribute, returns resident blocks per SM
constexpr int MV_SHAPES = 2;  // ring shapes of the staged FP32 matvec (option staged_matvec 1..2)

struct CellOcc {
    int p_update, s_update, xr_update, matvec, matvec_pair, copy, outer;
    int matvec_staged[MV_SHAPES + 1];  // the bulk-copy staged FP32 matvec, per ring shape 1.. (0: it cannot run)
};
void cell_occupancy(bool fp32, CellOcc *o);

// ---- the gas pressure-correction system assembled on the device
// (CONV_PP_G + SOURCE_PP_G, pp_assembly.cu); every pointer is device memory in
// the reference's layouts: cell arrays of DIMENSION_3, D_E(DIMENSION_3, 0:MMAX),
// ROP_SE etc. (DIMENSION_3, 1:MMAX) with phase m at m*n and (m-1)*n.
struct PPFields {
    const int *flag;  // FLAG: 1 fluid (FLUID_AT), 10/11 pressure inflow/outflow (P_FLOW_AT)
    const double *rop_ge, *rop_gn, *rop_gt, *ayz, *axz, *axy, *u_g, *v_g, *w_g;
    const double *rop_g, *rop_go, *vol, *sum_r_g, *d_e, *d_n, *d_t;
    int mmax;
    const int *close_packed;  // device copy of CLOSE_PACKED(1:MMAX)
    const double *rop_se, *rop_sn, *rop_st, *u_s, *v_s, *w_s, *rop_s, *rop_so, *sum_r_s;
    double odt;
    long long ijk_p_g;  // 1-based, <= 0: undefined
};
struct PPGeom {
    int imax2, jmax2, kmax2, do_k;
    int64_t n;
};
// A_M(:,:,0) (7n), B_M(:,0), B_MMAX(:,0) on the device
cudaError_t launch_conv_source_pp(const PPFields &f, const PPGeom &g, double *a, double *b, double *bmmax, int grid,
                                  cudaStream_t s);
// CALC_RESID_PP's RESID of v over the fluid cells with normalization norm
// (blocks' partial sums in part_dev, 2 * grid doubles); synchronizes the stream.
cudaError_t resid_pp(const int *flag, const double *v, int64_t n, double norm, double *part_dev, int grid,
                     cudaStream_t s, double *resid);

}  // namespace mfixgpu
