// pp_assembly.cu -- the gas pressure-correction system assembled on the device:
// CONV_PP_G (model/conv_pp_g.f:33-182) and SOURCE_PP_G (model/source_pp_g.f:18-214)
// for an incompressible run on a Cartesian grid without shear, and the
// residual of CALC_RESID_PP (model/calc_resid.f:391-534).  SOLVE_PP_G
// (model/solve_pp_g.f:10-118) then hands A_M(:,:,0) / B_M(:,0) to SOLVE_LIN_EQ
// without the arrays ever crossing the host link.
//
// CONV_PP_G writes each face coefficient from the cell below the face
// (ROP_GE(IJK)*AYZ(IJK) becomes A_M(IJK,east) and A_M(IP_OF(IJK),west)); here each
// fluid cell gathers its six: A(west) = ROP_GE(IMJK)*AYZ(IMJK) whether or not
// IMJK is fluid (:80-106), so one thread per cell and no write conflicts.  Every
// product and sum is rounded separately in the reference's left-to-right order
// (__dmul_rn / __dadd_rn: no fused multiply-adds), so the system is bit for bit
// the one the reference's Fortran (compiled without FMA contraction) builds.
#include <cmath>
#include <vector>

#include "leq_kernels.cuh"

namespace mfixgpu {

namespace {

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

__device__ __forceinline__ bool fluid_at(const int *flag, int64_t p) { return flag[p] == 1; }
__device__ __forceinline__ bool p_flow_at(const int *flag, int64_t p) { return flag[p] == 10 || flag[p] == 11; }

__global__ void __launch_bounds__(256) k_conv_source_pp(PPFields f, PPGeom g, double *a, double *b, double *bmmax)
{
    const int64_t n = g.n, c1 = g.jmax2, c2 = (int64_t)g.jmax2 * g.imax2;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
        if (!fluid_at(f.flag, p)) {  // wall and flow-boundary cells: identity rows (:187-199)
            for (int q = 0; q < 7; ++q) a[q * n + p] = q == 3 ? -1.0 : 0.0;
            b[p] = 0.0;
            bmmax[p] = 0.0;
            continue;
        }
        const int64_t line = p / g.jmax2;
        const int j = (int)(p - line * g.jmax2);
        const int k = (int)(line / g.imax2);
        const int i = (int)(line - (int64_t)k * g.imax2);
        // clamped neighbours (model/set_increments.f:80-109)
        const int64_t im = p + (i > 0 ? -c1 : 0), ip = p + (i < g.imax2 - 1 ? c1 : 0);
        const int64_t jm = p + (j > 0 ? -1 : 0), jp = p + (j < g.jmax2 - 1 ? 1 : 0);
        const int64_t km = p + ((g.do_k && k > 0) ? -c2 : 0), kp = p + ((g.do_k && k < g.kmax2 - 1) ? c2 : 0);
        // CONV_PP_G, gas phase (:80-119)
        double ae = mul(f.rop_ge[p], f.ayz[p]);
        double aw = mul(f.rop_ge[im], f.ayz[im]);
        double an = mul(f.rop_gn[p], f.axz[p]);
        double as = mul(f.rop_gn[jm], f.axz[jm]);
        double at = 0.0, ab = 0.0;
        if (g.do_k) {
            at = mul(f.rop_gt[p], f.axy[p]);
            ab = mul(f.rop_gt[km], f.axy[km]);
        }
        // SOURCE_PP_G (:87-106)
        const double bma = mul(mul(sub(f.rop_g[p], f.rop_go[p]), f.vol[p]), f.odt);
        const double bme = mul(ae, f.u_g[p]);
        const double bmw = mul(aw, f.u_g[im]);
        const double bmn = mul(an, f.v_g[p]);
        const double bms = mul(as, f.v_g[jm]);
        const double bmt = g.do_k ? mul(at, f.w_g[p]) : 0.0;
        const double bmb = g.do_k ? mul(ab, f.w_g[km]) : 0.0;
        const double bmr = mul(f.sum_r_g[p], f.vol[p]);
        const double inner = sub(add(sub(add(sub(add(bma, bme), bmw), bmn), bms), bmt), bmb);
        double bv = -(add(-inner, bmr));
        double mx = fabs(bma);
        mx = fmax(mx, fabs(bme));
        mx = fmax(mx, fabs(bmw));
        mx = fmax(mx, fabs(bmn));
        mx = fmax(mx, fabs(bms));
        mx = fmax(mx, fabs(bmt));
        mx = fmax(mx, fabs(bmb));
        mx = fmax(mx, fabs(bmr));
        ae = mul(ae, f.d_e[p]);
        aw = mul(aw, f.d_e[im]);
        an = mul(an, f.d_n[p]);
        as = mul(as, f.d_n[jm]);
        if (g.do_k) {
            at = mul(at, f.d_t[p]);
            ab = mul(ab, f.d_t[km]);
        }
        // solids phases that do not become close packed (:117-145; CONV_PP_G :125-178)
        for (int m = 1; m <= f.mmax; ++m) {
            if (f.close_packed[m - 1]) continue;
            const int64_t o = (int64_t)(m - 1) * n, od = (int64_t)m * n;
            const double se = mul(f.rop_se[o + p], f.ayz[p]);
            const double sw = mul(f.rop_se[o + im], f.ayz[im]);
            const double sn = mul(f.rop_sn[o + p], f.axz[p]);
            const double ss = mul(f.rop_sn[o + jm], f.axz[jm]);
            double st = 0.0, sb = 0.0;
            if (g.do_k) {
                st = mul(f.rop_st[o + p], f.axy[p]);
                sb = mul(f.rop_st[o + km], f.axy[km]);
            }
            const double wt = g.do_k ? mul(st, f.w_s[o + p]) : 0.0;
            const double wb = g.do_k ? mul(sb, f.w_s[o + km]) : 0.0;
            double t = mul(mul(sub(f.rop_s[o + p], f.rop_so[o + p]), f.vol[p]), f.odt);
            t = add(t, mul(se, f.u_s[o + p]));
            t = sub(t, mul(sw, f.u_s[o + im]));
            t = add(t, mul(sn, f.v_s[o + p]));
            t = sub(t, mul(ss, f.v_s[o + jm]));
            t = add(t, wt);
            t = sub(t, wb);
            bv = sub(bv, add(-t, mul(f.sum_r_s[o + p], f.vol[p])));
            ae = add(ae, mul(se, f.d_e[od + p]));
            aw = add(aw, mul(sw, f.d_e[od + im]));
            an = add(an, mul(sn, f.d_n[od + p]));
            as = add(as, mul(ss, f.d_n[od + jm]));
            if (g.do_k) {
                at = add(at, mul(st, f.d_t[od + p]));
                ab = add(ab, mul(sb, f.d_t[od + km]));
            }
        }
        double ac = -add(add(add(add(add(ae, aw), an), as), at), ab);  // :147-149
        if (fabs(ac) < 1.0e-15 && fabs(bv) < 1.0e-15) {                 // :151-162, SMALL_NUMBER
            ac = -1.0;
            bv = 0.0;
        }
        // links to pressure-flow cells cut (:224-243)
        if (p_flow_at(f.flag, im)) aw = 0.0;
        if (p_flow_at(f.flag, ip)) ae = 0.0;
        if (p_flow_at(f.flag, jm)) as = 0.0;
        if (p_flow_at(f.flag, jp)) an = 0.0;
        if (p_flow_at(f.flag, km)) ab = 0.0;
        if (p_flow_at(f.flag, kp)) at = 0.0;
        a[0 * n + p] = ab;  // A_M(IJK,-3) = bottom
        a[1 * n + p] = as;  // -2 south
        a[2 * n + p] = aw;  // -1 west
        a[3 * n + p] = ac;
        a[4 * n + p] = ae;  //  1 east
        a[5 * n + p] = an;  //  2 north
        a[6 * n + p] = at;  //  3 top
        b[p] = bv;
        bmmax[p] = mx;
    }
}

// the reference cell of an incompressible run (:247-251)
__global__ void k_pp_ref_cell(double *a, double *b, int64_t n, int64_t p)
{
    if (threadIdx.x < 7) a[threadIdx.x * n + p] = threadIdx.x == 3 ? -1.0 : 0.0;
    if (threadIdx.x == 0) b[p] = 0.0;
}

// CALC_RESID_PP's sums over the fluid cells: sum |v| and the cell count, per block
// (the host adds the blocks in order).
__global__ void __launch_bounds__(256) k_resid_pp(const int *flag, const double *v, int64_t n, double *part)
{
    __shared__ double s_num[256], s_den[256];
    double num = 0.0, den = 0.0;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x)
        if (flag[p] == 1) {
            num += fabs(v[p]);
            den += 1.0;
        }
    s_num[threadIdx.x] = num;
    s_den[threadIdx.x] = den;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            s_num[threadIdx.x] += s_num[threadIdx.x + s];
            s_den[threadIdx.x] += s_den[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = s_num[0];
        part[2 * blockIdx.x + 1] = s_den[0];
    }
}

}  // namespace

cudaError_t launch_conv_source_pp(const PPFields &f, const PPGeom &g, double *a, double *b, double *bmmax, int grid,
                                  cudaStream_t s)
{
    k_conv_source_pp<<<grid, 256, 0, s>>>(f, g, a, b, bmmax);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (f.ijk_p_g >= 1 && f.ijk_p_g <= g.n) {
        k_pp_ref_cell<<<1, 32, 0, s>>>(a, b, g.n, f.ijk_p_g - 1);
        e = cudaGetLastError();
    }
    return e;
}

cudaError_t resid_pp(const int *flag, const double *v, int64_t n, double norm, double *part_dev, int grid,
                     cudaStream_t s, double *resid)
{
    k_resid_pp<<<grid, 256, 0, s>>>(flag, v, n, part_dev);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    std::vector<double> h(2 * (size_t)grid);
    e = cudaMemcpyAsync(h.data(), part_dev, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return e;
    double num = 0.0, den = 0.0;
    for (int q = 0; q < grid; ++q) {
        num += h[2 * q];
        den += h[2 * q + 1];
    }
    // model/calc_resid.f:468-476
    if (den * norm > 0.0)
        *resid = num / (den * norm);
    else if (num == 0.0)
        *resid = 0.0;
    else
        *resid = 1.0e32;  // LARGE_NUMBER
    return cudaSuccess;
}

}  // namespace mfixgpu
