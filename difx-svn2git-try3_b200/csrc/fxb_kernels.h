// Kernel launchers (host-callable) of the sm_100a FX path.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "fxb_internal.h"

namespace fxb {

// Per-frequency XMAC plan on the device.
struct DevFreqPlan {
	int32_t nrow, nchan, ntr, npair;  // rows, channels, 4-row tiles, tile pairs
	int32_t r2pad;                    // real rows per channel of the K-major BF16 spectra (2*nrow rounded up to 8)
	int32_t tpad;                     // FFTs per subint rounded up to the K tile (64)
	int32_t acc_cstride;              // accumulator stride between channels (1: [out][chan], nout: [chan][out])
	int32_t acc_ostride;              // accumulator stride between outputs
	int64_t spec_off;                 // complex offset of spectra [T][nrow][nchan]
	int64_t acc_off;                  // complex offset of accumulators [nout][nchan]
	const int32_t *destA;             // [nrow*nrow]
	const int32_t *destB;             // [nrow*nrow]
	const int16_t *pairs;             // [npair*2] tile pairs (ti <= tj)
};

struct DevOutMap {
	int64_t acc, core;
	int32_t nchan, avg;
	int32_t cstride, pad;
};

struct DevBWeight {
	int32_t s1, s2;
	int64_t dst;
};

struct DevACWeight {
	int32_t s, pad;
	int64_t dst;
};

void launch_frame_valid(const DevStation *st, const DevSubintStation *sub, uint8_t *valid, int64_t valid_stride,
                        int S, cudaStream_t stream);
void launch_interpolators(const DevStation *st, DevSubintStation *sub, int S, int blockspersend, int sec, int ns,
                          cudaStream_t stream);
void launch_fft_params(const DevStation *st, const DevSubintStation *sub, const int32_t *validflags, int nflagint,
                       const uint8_t *valid, int64_t valid_stride, int S, int T, int sec, int ns, int order,
                       FftParam *out, cudaStream_t stream);

// Fused unpack -> fringe rotation -> FFT -> fractional-sample correction.
// One CTA per (station, FFT); writes FP32 spectra into spec.
void launch_fstage(const DevStation *st, const DevSubintStation *sub, const DevBand *bands, int maxband,
                   const DevFreqPlan *plans, const uint8_t *valid, int64_t valid_stride, const FftParam *params,
                   const float2 *twiddle, int maxN, int S, int T, int order, bool fractionallofreq, int maxfft,
                   float2 *spec, cudaStream_t stream);

// F stage v2 (csrc/fxb_fstage.cu): CTA per (station, subband, chunk of TQ FFTs).
// out 0: FP32 rows [t][row][chan]; out 1: BF16 K-major [chan][2 row + part][tpad].
void launch_fstage2(const DevStation *st, const DevSubintStation *sub, const void *groups, int npair, int nsingle,
                    const DevFreqPlan *plans, const uint8_t *valid, int64_t valid_stride, const FftParam *params,
                    const float2 *twiddle, int maxN, int T, int TQ, int Tpad, int order, bool fractionallofreq,
                    int N, int nband_max, int nbits_max, int nbufmax, int out, void *spec, cudaStream_t stream);
size_t fgroup_size();
void make_fgroup(void *dst, int station, int freq, int b0, int b1, int r0, int r1, int lsb, double lofreq);

// FP32 XMAC v2 over a set of frequencies with equal (rows, channels):
// plan_idx[0..nf) index dplans.
void launch_xmac_fp32v2(const DevFreqPlan &plan0, const DevFreqPlan *dplans, const int32_t *plan_idx, int nf, int T,
                        const float2 *spec, float2 *acc, cudaStream_t stream);

// Tensor-core XMAC (csrc/fxb_xmac_tc.cu).
bool tc_make_tensormap(void *map_out, const void *spec_bf16, int64_t total_rows, int Tpad, int boxrows);
size_t tc_tensormap_size();
void tc_geometry(int R2, int Tpad, int *G, int *NG, int *boxrows, int *tmem_cols, size_t *smem);
void launch_xmac_tc(const void *tmap, const DevFreqPlan *dplans, const int32_t *plan_idx, int nf, int nchan,
                    const int64_t *rowbase, int Tpad, int R2, int32_t *err, float2 *acc, cudaStream_t stream);

// FP32 cross-multiply-accumulate of one frequency into acc.
void launch_xmac_fp32(const DevFreqPlan &plan, const DevFreqPlan *dplan, int T, const float2 *spec, float2 *acc,
                      cudaStream_t stream);

void launch_weights(const DevBWeight *bw, int nbw, const DevACWeight *acw, int nacw, const FftParam *params, int T,
                    float *bwacc, float *acwacc, cudaStream_t stream);

void launch_finalise(const DevOutMap *om, int nom, int maxout, const float2 *acc, const DevBWeight *bw, int nbw,
                     const float *bwacc, const DevACWeight *acw, int nacw, const float *acwacc, float2 *core,
                     int64_t corelen, cudaStream_t stream);

void launch_vdif_unpack(const uint8_t *data, int64_t nbytes, int payload, int header, int nchan, int nbits,
                        int64_t offsetsamples, int nsamp, float *out, int *good, cudaStream_t stream);

}  // namespace fxb
