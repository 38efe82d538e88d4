// tcs_fields.cuh -- the device-resident state of one case and the small
// helpers the stage kernels share.
#pragma once

#include "tcs_device.cuh"

namespace tcs {

template <class R>
struct FieldsT {
    // persistent fields (padded, i fastest)
    R *T, *U, *V, *W, *P, *dPhat, *dP0;
    // second buffers of the fields that a kernel rewrites while other threads
    // still read the old values (T in the thermal y sweep, U/V/W in the fused
    // pseudo-update, dPhat/dP0 in the projection)
    R *Tn, *Un, *Vn, *Wn, *dPhatn, *dP0n;
    // per-step increments and pressure correction
    R *dU, *dV, *dW, *dP;
    // interior stage scratch (padded layout)
    R *scr;
    // 2-D (j,k) property tables: Mu and invRho of mpi_momentum_coeffi
    R *Mu2, *iR2;
    // Poisson spectral work array: (h1p, N2, N3) complex, kx fastest
    cplx_t<R> *S;
    // modified wavenumbers and y coefficients of the modal solves (FP64 in both forms)
    const double *dxk2, *dzk, *fam, *fap;
    // FFT twiddles exp(-2 pi i e / n) for n = N1 and n = N3
    const cplx_t<R> *tw1, *tw3;
    // reduction scratch
    double *part;
    double *hist;            // per-step diagnostics history (7 doubles per step)
    int hist_cap;
};

// Skip all work once the divergence check has flagged a blow-up, so the
// fields stay at the state of the step that blew up (main.f90:208-212).
template <class R>
__device__ __forceinline__ bool blown(const GridT<R> &g) { return g.scal[S_BLOWUP] != 0.0; }

} // namespace tcs
