// tcs_post.cu -- per-step diagnostics: mpi_Post_Div and mpi_Post_CFL
// (module_post.f90:100-158, 168-230) with the adaptive time step, the
// blow-up test of main.f90:208-212, and the Nusselt / kinetic-energy series.
// Two kernels: block partials in a fixed order, then one block that combines
// them and updates dt, time and CFL on the device (deterministic).  Both forms
// reduce in FP64 from their fields, and the per-thread sums are compensated
// (Neumaier), so the diagnostics keep FP64 accuracy over 512^3 cells.
#include "tcs_kernels.h"

#include <math.h>

namespace tcs {

enum { PT_DIV = 0, PT_CFL, PT_KE, PT_NUB, PT_NUT, PT_N };
static const int POST_BLOCKS = 592;   // 4 x 148 SMs

// s + e carries a sum and its running rounding error (Neumaier's variant of
// Kahan summation).
__device__ __forceinline__ void csum(double &s, double &e, double v)
{
    const double t = s + v;
    e += (fabs(s) >= fabs(v)) ? (s - t) + v : (v - t) + s;
    s = t;
}

template <class R>
__global__ void __launch_bounds__(256) post_kernel(GridT<R> g, FieldsT<R> f, FastDiv dn1, FastDiv dn2)
{
    __shared__ double red[PT_N][256];
    if (blown(g)) return;
    const long long n = (long long)g.N1 * g.N2 * g.N3;
    double mdiv = -INFINITY, mcfl = -INFINITY, ke = 0.0, nub = 0.0, nut = 0.0, eke = 0.0, enb = 0.0, ent = 0.0;
    const double *dx1 = g.d1.dx, *dx2 = g.d2.dx, *dx3 = g.d3.dx;
    const double *rdx1 = g.d1.rdx, *rdx2 = g.d2.rdx, *rdx3 = g.d3.rdx;
    const long long sj = g.P1, sk = (long long)g.P1 * g.P2;
    // two cells per pass keep twice the loads in flight (measured -21% at 256^3)
#pragma unroll 2
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const unsigned q = dn1.div((unsigned)t), r = dn2.div(q);     // n < 2^31: 32-bit multiply-shift division
        const int i = 1 + (int)((unsigned)t - q * (unsigned)g.N1);
        const int j = 1 + (int)(q - r * (unsigned)g.N2), k = 1 + (int)r;
        const long long c = ix(g, i, j, k);
        double Uc, Vc, Wc, Ux, Vy, Wz;
        if constexpr (HasLo<R>::on) {     // the FP32 form's velocity is its high + low pair
            Uc = join(ld(f.U + c), ld(f.Ulo + c)); Vc = join(ld(f.V + c), ld(f.Vlo + c)); Wc = join(ld(f.W + c), ld(f.Wlo + c));
            Ux = join(ld(f.U + c + 1), ld(f.Ulo + c + 1)); Vy = join(ld(f.V + c + sj), ld(f.Vlo + c + sj));
            Wz = join(ld(f.W + c + sk), ld(f.Wlo + c + sk));
        } else {
            Uc = ld(f.U + c); Vc = ld(f.V + c); Wc = ld(f.W + c);
            Ux = ld(f.U + c + 1); Vy = ld(f.V + c + sj); Wz = ld(f.W + c + sk);
        }
        const double dv = (Ux - Uc) * rdx1[i] + (Vy - Vc) * rdx2[j] + (Wz - Wc) * rdx3[k];
        const double cf = (fabs(Ux + Uc) / 2.0) * rdx1[i] + (fabs(Vy + Vc) / 2.0) * rdx2[j] + (fabs(Wz + Wc) / 2.0) * rdx3[k];
        mdiv = fmax(mdiv, dv);
        mcfl = fmax(mcfl, cf);
        csum(ke, eke, (Uc * Uc + Vc * Vc + Wc * Wc) * dx1[i] * dx2[j] * dx3[k]);
        if (j == 1) csum(nub, enb, -((double)ld(f.T + c) - g.phd.Tbt) / g.d2.dmx[1]);
        if (j == g.N2) csum(nut, ent, -(g.phd.Tup - (double)ld(f.T + c)) / g.d2.dmx[g.N2 + 1]);
    }
    ke += eke; nub += enb; nut += ent;
    red[PT_DIV][threadIdx.x] = mdiv; red[PT_CFL][threadIdx.x] = mcfl;
    red[PT_KE][threadIdx.x] = ke; red[PT_NUB][threadIdx.x] = nub; red[PT_NUT][threadIdx.x] = nut;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            red[PT_DIV][threadIdx.x] = fmax(red[PT_DIV][threadIdx.x], red[PT_DIV][threadIdx.x + w]);
            red[PT_CFL][threadIdx.x] = fmax(red[PT_CFL][threadIdx.x], red[PT_CFL][threadIdx.x + w]);
            red[PT_KE][threadIdx.x] += red[PT_KE][threadIdx.x + w];
            red[PT_NUB][threadIdx.x] += red[PT_NUB][threadIdx.x + w];
            red[PT_NUT][threadIdx.x] += red[PT_NUT][threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x < PT_N) f.part[blockIdx.x * PT_N + threadIdx.x] = red[threadIdx.x][0];
}

template <class R>
__global__ void __launch_bounds__(256) finalize_kernel(GridT<R> g, FieldsT<R> f, int nblocks, int record_hist)
{
    __shared__ double red[PT_N][256];
    if (blown(g)) return;
    double mdiv = -INFINITY, mcfl = -INFINITY, ke = 0.0, nub = 0.0, nut = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
        const double *p = f.part + b * PT_N;
        mdiv = fmax(mdiv, p[PT_DIV]); mcfl = fmax(mcfl, p[PT_CFL]);
        ke += p[PT_KE]; nub += p[PT_NUB]; nut += p[PT_NUT];
    }
    red[PT_DIV][threadIdx.x] = mdiv; red[PT_CFL][threadIdx.x] = mcfl;
    red[PT_KE][threadIdx.x] = ke; red[PT_NUB][threadIdx.x] = nub; red[PT_NUT][threadIdx.x] = nut;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            red[PT_DIV][threadIdx.x] = fmax(red[PT_DIV][threadIdx.x], red[PT_DIV][threadIdx.x + w]);
            red[PT_CFL][threadIdx.x] = fmax(red[PT_CFL][threadIdx.x], red[PT_CFL][threadIdx.x + w]);
            red[PT_KE][threadIdx.x] += red[PT_KE][threadIdx.x + w];
            red[PT_NUB][threadIdx.x] += red[PT_NUB][threadIdx.x + w];
            red[PT_NUT][threadIdx.x] += red[PT_NUT][threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    double *sc = g.scal;
    const double dt_used = sc[S_DT];
    const double maxdiv = red[PT_DIV][0], mx = red[PT_CFL][0];
    const double cnt = (double)g.N1 * (double)g.N3;
    sc[S_MAXDIV] = maxdiv;
    sc[S_NUBOT] = red[PT_NUB][0] / cnt;
    sc[S_NUTOP] = red[PT_NUT][0] / cnt;
    sc[S_KE] = 0.5 * red[PT_KE][0] / (g.phd.L1 * g.phd.L2 * g.phd.L3);
    if (maxdiv >= 1.0e-3 || maxdiv != maxdiv) {
        sc[S_BLOWUP] = sc[S_STEP] + 1.0;          // the step (1-based) that blew up
        return;
    }
    if (sc[S_FIXED_DT] != 0.0) {
        sc[S_CFL] = dt_used * mx;
    } else {
        double nd = g.phd.MaxCFL / mx;              // +Inf for a resting fluid
        if (nd > g.phd.dtMax) nd = g.phd.dtMax;
        sc[S_DT] = nd;
        sc[S_CFL] = nd * mx;
    }
    sc[S_TIME] = sc[S_TIME] + sc[S_DT];
    const int step = (int)sc[S_STEP];
    if (record_hist && step < f.hist_cap) {
        double *h = f.hist + (long long)step * 7;
        h[0] = dt_used; h[1] = sc[S_TIME]; h[2] = maxdiv; h[3] = sc[S_CFL];
        h[4] = sc[S_NUBOT]; h[5] = sc[S_NUTOP]; h[6] = sc[S_KE];
    }
    sc[S_STEP] = step + 1;
}

template <class R>
void launch_post(const Ctx<R> &cx, cudaStream_t s, int record_hist)
{
    probe_begin(cx, K_POST, s);
    post_kernel<<<POST_BLOCKS, 256, 0, s>>>(cx.g, cx.f, make_fastdiv((unsigned)cx.g.N1), make_fastdiv((unsigned)cx.g.N2));
    probe_end(cx, K_POST, s);
    record_launch_error("post");
    probe_begin(cx, K_FINAL, s);
    finalize_kernel<<<1, 256, 0, s>>>(cx.g, cx.f, POST_BLOCKS, record_hist);
    probe_end(cx, K_FINAL, s);
    record_launch_error("finalize");
}

int post_partial_count() { return POST_BLOCKS * PT_N; }

// Periodic ghost update of one padded field (module_mpi_subdomain.f90:758-791):
// x faces first, then z faces including the x-ghost columns.
template <class R>
__global__ void ghost_x_kernel(GridT<R> g, R *a)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
    if (j > g.N2 + 1) return;
    a[ix(g, 0, j, k)] = a[ix(g, g.N1, j, k)];
    a[ix(g, g.N1 + 1, j, k)] = a[ix(g, 1, j, k)];
}
template <class R>
__global__ void ghost_z_kernel(GridT<R> g, R *a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (i > g.N1 + 1) return;
    a[ix(g, i, j, 0)] = a[ix(g, i, j, g.N3)];
    a[ix(g, i, j, g.N3 + 1)] = a[ix(g, i, j, 1)];
}

template <class R>
void launch_ghost(const Ctx<R> &cx, R *a, cudaStream_t s)
{
    const GridT<R> &g = cx.g;
    ghost_x_kernel<<<dim3((g.N2 + 2 + 127) / 128, g.N3 + 2), 128, 0, s>>>(g, a);
    ghost_z_kernel<<<dim3((g.N1 + 2 + 127) / 128, g.N2 + 2), 128, 0, s>>>(g, a);
    record_launch_error("ghost");
}

// Conversions between an FP32 field and an FP64 staging copy (the host API
// moves FP64 arrays in both forms).
template <class R>
__global__ void convert_out_kernel(const R *src, double *dst, long long n)
{
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) dst[t] = (double)src[t];
}
template <class R>
__global__ void convert_in_kernel(const double *src, R *dst, long long n)
{
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) dst[t] = (R)src[t];
}

// FP64 staging <-> FP32 high/low pair (the FP32 form's velocity).
__global__ void join_kernel(const float *hi, const float *lo, double *dst, long long n)
{
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) dst[t] = join(hi[t], lo[t]);
}
__global__ void split_kernel(const double *src, float *hi, float *lo, long long n)
{
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        float h, l;
        split(src[t], h, l);
        hi[t] = h; lo[t] = l;
    }
}

void launch_join(const float *hi, const float *lo, double *dst, long long n, cudaStream_t s)
{
    join_kernel<<<4 * 148, 256, 0, s>>>(hi, lo, dst, n);
    record_launch_error("join");
}
void launch_split(const double *src, float *hi, float *lo, long long n, cudaStream_t s)
{
    split_kernel<<<4 * 148, 256, 0, s>>>(src, hi, lo, n);
    record_launch_error("split");
}

template <class R>
void launch_convert(const R *src, double *dst, long long n, cudaStream_t s)
{
    convert_out_kernel<R><<<4 * 148, 256, 0, s>>>(src, dst, n);
    record_launch_error("convert_out");
}
template <class R>
void launch_convert_in(const double *src, R *dst, long long n, cudaStream_t s)
{
    convert_in_kernel<R><<<4 * 148, 256, 0, s>>>(src, dst, n);
    record_launch_error("convert_in");
}

// Interior k-slabs of a field to/from a packed FP64 array (i fastest), the
// layout of the reference's continue files (module_post.f90:1264-1454); in the
// FP32 form the velocity's low word is added on the way out and split off on
// the way in.
template <class R>
__global__ void pack_kernel(GridT<R> g, const R *src, const R *lo, double *dst, int k0, int nk)
{
    const int n = g.N1 * g.N2 * nk;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const int i = t % g.N1, q = t / g.N1, j = q % g.N2, k = q / g.N2;
        const long long c = ix(g, 1 + i, 1 + j, k0 + k);
        dst[t] = lo ? (double)src[c] + (double)lo[c] : (double)src[c];
    }
}
template <class R>
__global__ void unpack_kernel(GridT<R> g, const double *src, R *dst, R *dst2, R *lo, int k0, int nk)
{
    const int n = g.N1 * g.N2 * nk;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const int i = t % g.N1, q = t / g.N1, j = q % g.N2, k = q / g.N2;
        const long long c = ix(g, 1 + i, 1 + j, k0 + k);
        const R h = (R)src[t];
        dst[c] = h;
        if (dst2) dst2[c] = h;
        if (lo) lo[c] = (R)(src[t] - (double)h);
    }
}
// One padded plane of a field: axis 1 (i = index) over (j, k), axis 2 over
// (i, k), axis 3 over (i, j); the first of the two remaining indices fastest.
template <class R>
__global__ void plane_kernel(GridT<R> g, const R *src, const R *lo, double *dst, int axis, int index)
{
    const int P3 = g.N3 + 2;
    const int na = axis == 1 ? g.P2 : g.P1, nb = axis == 3 ? g.P2 : P3;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < na * nb; t += gridDim.x * blockDim.x) {
        const int a = t % na, b = t / na;
        const long long c = axis == 1 ? ix(g, index, a, b) : (axis == 2 ? ix(g, a, index, b) : ix(g, a, b, index));
        dst[t] = lo ? (double)src[c] + (double)lo[c] : (double)src[c];
    }
}

template <class R>
void launch_pack(const Ctx<R> &cx, const R *src, const R *lo, double *dst, int k0, int nk, cudaStream_t s)
{
    pack_kernel<R><<<4 * 148, 256, 0, s>>>(cx.g, src, lo, dst, k0, nk);
    record_launch_error("pack");
}
template <class R>
void launch_unpack(const Ctx<R> &cx, const double *src, R *dst, R *dst2, R *lo, int k0, int nk, cudaStream_t s)
{
    unpack_kernel<R><<<4 * 148, 256, 0, s>>>(cx.g, src, dst, dst2, lo, k0, nk);
    record_launch_error("unpack");
}
template <class R>
void launch_plane(const Ctx<R> &cx, const R *src, const R *lo, double *dst, int axis, int index, cudaStream_t s)
{
    plane_kernel<R><<<148, 256, 0, s>>>(cx.g, src, lo, dst, axis, index);
    record_launch_error("plane");
}

template void launch_pack<double>(const Ctx<double> &, const double *, const double *, double *, int, int, cudaStream_t);
template void launch_pack<float>(const Ctx<float> &, const float *, const float *, double *, int, int, cudaStream_t);
template void launch_unpack<double>(const Ctx<double> &, const double *, double *, double *, double *, int, int, cudaStream_t);
template void launch_unpack<float>(const Ctx<float> &, const double *, float *, float *, float *, int, int, cudaStream_t);
template void launch_plane<double>(const Ctx<double> &, const double *, const double *, double *, int, int, cudaStream_t);
template void launch_plane<float>(const Ctx<float> &, const float *, const float *, double *, int, int, cudaStream_t);

// the two forms
template void launch_post<double>(const Ctx<double> &, cudaStream_t, int);
template void launch_post<float>(const Ctx<float> &, cudaStream_t, int);
template void launch_ghost<double>(const Ctx<double> &, double *, cudaStream_t);
template void launch_ghost<float>(const Ctx<float> &, float *, cudaStream_t);
template void launch_convert<double>(const double *, double *, long long, cudaStream_t);
template void launch_convert<float>(const float *, double *, long long, cudaStream_t);
template void launch_convert_in<double>(const double *, double *, long long, cudaStream_t);
template void launch_convert_in<float>(const double *, float *, long long, cudaStream_t);

} // namespace tcs
