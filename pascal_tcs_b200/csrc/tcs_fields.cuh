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
    // FP32 form only: low words of the velocity (U = U + Ulo to FP64 accuracy)
    // and of its second buffers.  The stencils read the FP32 high word; the
    // pressure right-hand side, the projection and the diagnostics read both,
    // so the storage rounding of the velocity never reaches the divergence.
    R *Ulo, *Vlo, *Wlo, *Unlo, *Vnlo, *Wnlo;
    // per-step increments and pressure correction
    R *dU, *dV, *dW, *dP;
    // interior stage scratch (padded layout)
    R *scr;
    // the pressure right-hand side of the split form (FP64, padded layout): the
    // FP64 form's scr, the FP32 form's FP64 staging array; null where the split
    // form does not run
    double *prhs;
    // 2-D (j,k) property tables: Mu and invRho of mpi_momentum_coeffi, in the
    // field type (read by the line sweeps), and invRho in FP64 (the same array
    // in the FP64 form).  invRho differs from 1 by about 1e-3 for water, and
    // the pressure right-hand side and the projection use 1 - invRho: from an
    // FP32 table those terms carried 6e-5 relative error, which left P 2-3e-5
    // off the FP64 form after 5-8 steps of the 256^3 and 512^3 water cases
    // (3-8e-6 with the FP64 table).
    R *Mu2, *iR2;
    double *iR2d;
    // Poisson spectral work array: (h1p, N2, N3) complex, kx fastest
    cplx_t<R> *S;
    // modified wavenumbers and y coefficients of the modal solves (FP64 in both forms)
    const double *dxk2, *dzk, *fam, *fap;
    // FFT twiddles exp(-2 pi i e / n) for n = N1 and n = N3 (FFT arithmetic is FP64 in both forms)
    const double2 *tw1, *tw3;
    // reduction scratch
    double *part;
    double *hist;            // per-step diagnostics history (7 doubles per step)
    int hist_cap;
};

// Skip all work once the divergence check has flagged a blow-up, so the
// fields stay at the state of the step that blew up (main.f90:208-212).
template <class R>
__device__ __forceinline__ bool blown(const GridT<R> &g) { return g.scal[S_BLOWUP] != 0.0; }

// The FP32 form keeps low words of the velocity.
template <class R> struct HasLo { static constexpr bool on = std::is_same<R, float>::value; };

// v = hi + lo in FP64, and its split back into an FP32 pair.
__device__ __forceinline__ double join(float hi, float lo) { return (double)hi + (double)lo; }
__device__ __forceinline__ void split(double v, float &hi, float &lo)
{
    hi = (float)v;
    lo = (float)(v - (double)hi);
}

} // namespace tcs
