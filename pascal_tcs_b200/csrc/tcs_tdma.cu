// tcs_tdma.cu -- the PaScaL_TDMA many-systems interface on one GPU:
// PaScaL_TDMA_many_solve and PaScaL_TDMA_many_solve_cycle
// (pascal_tdma.f90:487-578, 715-806) for one rank, with the reduced 2-row
// systems of tdma_many / tdma_cycl_many (tdmas.f90:113-146, 159-212).
//
// Arrays are the reference's (n_sys, n_row) with the system index fastest,
// so one thread per system reads and writes fully coalesced rows.  The
// arithmetic is the reference's, operation for operation, with explicit
// round-to-nearest intrinsics so that no multiply-add is fused: the results
// are bit-identical to a strict IEEE evaluation of the Fortran expressions
// (including the one-rank cyclic closure, where e(2) = -a(2) is overwritten by
// e(n2) = -c(2)).  D receives the solution; A and C are clobbered as in the
// reference.
#include "tcs_kernels.h"

namespace tcs {

#define MUL(a, b) __dmul_rn((a), (b))
#define SUB(a, b) __dsub_rn((a), (b))
#define ADD(a, b) __dadd_rn((a), (b))
#define DIV(a, b) __ddiv_rn((a), (b))

__global__ void tdma_many_kernel(double *__restrict__ A, const double *__restrict__ B, double *__restrict__ C,
                                 double *__restrict__ D, int n_sys, int n_row, int cyclic)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_sys) return;
    const size_t s = (size_t)n_sys;
#define a(j) A[(size_t)i + s * (size_t)(j)]
#define b(j) B[(size_t)i + s * (size_t)(j)]
#define c(j) C[(size_t)i + s * (size_t)(j)]
#define d(j) D[(size_t)i + s * (size_t)(j)]
    double r;
    a(0) = DIV(a(0), b(0)); d(0) = DIV(d(0), b(0)); c(0) = DIV(c(0), b(0));
    a(1) = DIV(a(1), b(1)); d(1) = DIV(d(1), b(1)); c(1) = DIV(c(1), b(1));
    double am1 = a(1), cm1 = c(1), dm1 = d(1);
    for (int j = 2; j < n_row; j++) {
        const double aj = a(j);
        r = DIV(1.0, SUB(b(j), MUL(aj, cm1)));
        dm1 = MUL(r, SUB(d(j), MUL(aj, dm1))); d(j) = dm1;
        cm1 = MUL(r, c(j)); c(j) = cm1;
        am1 = MUL(MUL(-r, aj), am1); a(j) = am1;
    }
    if (n_row >= 3) {
        double ap1 = a(n_row - 2), cp1 = c(n_row - 2), dp1 = d(n_row - 2);
        for (int j = n_row - 3; j >= 1; j--) {
            const double cj = c(j);
            dp1 = SUB(d(j), MUL(cj, dp1)); d(j) = dp1;
            ap1 = SUB(a(j), MUL(cj, ap1)); a(j) = ap1;
            cp1 = MUL(-cj, cp1); c(j) = cp1;
        }
    }
    r = DIV(1.0, SUB(1.0, MUL(a(1), c(0))));
    d(0) = MUL(r, SUB(d(0), MUL(c(0), d(1))));
    a(0) = MUL(r, a(0));
    c(0) = MUL(MUL(-r, c(0)), c(1));
    const double A1 = a(0), C1 = c(0), D1 = d(0);
    const double A2 = a(n_row - 1), C2 = c(n_row - 1), D2 = d(n_row - 1);
    double x1, x2;
    if (cyclic) {
        const double e2 = -C2;
        x1 = DIV(SUB(SUB(D1, MUL(A1, D2)), MUL(C1, D2)), ADD(ADD(1.0, MUL(A1, e2)), MUL(C1, e2)));
        x2 = ADD(D2, MUL(x1, e2));
    } else {
        r = DIV(1.0, SUB(1.0, MUL(A2, C1)));
        x2 = MUL(r, SUB(D2, MUL(A2, D1)));
        x1 = SUB(D1, MUL(C1, x2));
    }
    d(0) = x1;
    d(n_row - 1) = x2;
    for (int j = 1; j < n_row - 1; j++) d(j) = SUB(SUB(d(j), MUL(a(j), x1)), MUL(c(j), x2));
#undef a
#undef b
#undef c
#undef d
}

#undef MUL
#undef SUB
#undef ADD
#undef DIV

void launch_tdma_many(double *A, const double *B, double *C, double *D, int n_sys, int n_row, int cyclic, cudaStream_t s)
{
    tdma_many_kernel<<<(n_sys + 127) / 128, 128, 0, s>>>(A, B, C, D, n_sys, n_row, cyclic);
    record_launch_error("tdma_many");
}

} // namespace tcs
