// Kernel launchers (host-callable) of the sm_100a FX path.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "fxb_internal.h"

namespace fxb {

// Per-frequency XMAC plan on the device.
struct DevFreqPlan {
	int32_t nrow, nchan, ntr, npair;  // rows, channels, 4-row tiles, tile pairs
	int32_t tcb;                      // tensor-core form: channels per spectra block (0: spectra [t][row][chan])
	int32_t tnblk;                    // tensor-core form: blocks per time, spectra [t][block][row][tcb]
	int32_t acc_cstride;              // accumulator stride between channels (1: [out][chan], nout: [chan][out])
	int32_t acc_ostride;              // accumulator stride between outputs
	int64_t spec_off;                 // complex offset of this frequency's spectra
	int64_t acc_off;                  // complex offset of accumulators [nout][nchan]
	const int32_t *destA;             // [nrow*nrow]
	const int32_t *destB;             // [nrow*nrow]
	const int16_t *pairs;             // [npair*2] tile pairs (ti <= tj)
	const int32_t *outsrc;            // [nout] source of each output: a | b << 8 | conj << 16 (a <= b), or -1
	int64_t spec8_off;                // FP8 form: offset (16-bit words) of this frequency's e4m3 spectra
	float *iscale;                    // FP8 form: [nchan][nrow] 1 / quantisation scale of the subint
};

struct DevOutMap {
	int64_t acc, core;
	int32_t nchan, avg;
	int32_t cstride, pad;
};

struct DevBWeight {
	int32_t s1, s2, b1, b2;   // stations and recorded bands
	int64_t dst;
};

struct DevACWeight {
	int32_t s, band;          // station and band (per-band weights of INTERLACEDVDIF stations)
	int64_t dst;
};

// One zoom-band row: spectra channels [choff, choff + nchan) of row src_row
// of plan src_plan, copied to row dst_row of plan dst_plan.
struct DevZoomCopy {
	int32_t src_plan, src_row, dst_plan, dst_row, choff, nchan;
};

// raw INTERLACEDVDIF reads (DevStation::muxraw): frame slots, muxed headers
// and the muxed stream's length and start, before the frame validity
// (fxb_mux.cu); maxslots / maxproc bound every raw station's slots / frames
void launch_mux_raw(const DevStation *st, DevSubintStation *sub, int S, int maxslots, int maxproc,
                    cudaStream_t stream);
// bandok (may be null): per frame, the bands that keep their samples
// fillok (may be null): per frame, no fill pattern (the only check that the
// first frame of a complex unpack window gets)
void launch_frame_valid(const DevStation *st, const DevSubintStation *sub, uint8_t *valid, uint32_t *bandok,
                        int64_t valid_stride, int S, cudaStream_t stream, uint8_t *fillok = nullptr);
// the subint time is read from sub[s].subsec / subns
void launch_interpolators(const DevStation *st, DevSubintStation *sub, int S, int blockspersend, cudaStream_t stream);
// launch_interpolators and launch_frame_valid as one launch (stations without
// raw INTERLACEDVDIF reads, whose frame check needs the placement first)
void launch_prep(const DevStation *st, DevSubintStation *sub, int S, int blockspersend, uint8_t *valid,
                 uint32_t *bandok, int64_t valid_stride, cudaStream_t stream, uint8_t *fillok);
void launch_fft_params(const DevStation *st, const DevSubintStation *sub, const int32_t *validflags, int nflagint,
                       const uint8_t *valid, const uint32_t *bandok, int64_t valid_stride, int S, int T, int order,
                       FftParam *out, float *pbw, int nbm, cudaStream_t stream, const uint8_t *fillok = nullptr);

// Fused unpack -> fringe rotation -> FFT -> fractional-sample correction.
// One CTA per (station, FFT); writes FP32 spectra into spec.  Returns the
// launch's error (including that of raising the shared-memory limit).
cudaError_t launch_fstage(const DevStation *st, const DevSubintStation *sub, const DevBand *bands, int maxband,
                   const DevFreqPlan *plans, const uint8_t *valid, int64_t valid_stride, const FftParam *params,
                   const float2 *twiddle, int maxN, int S, int T, int order, bool fractionallofreq, int maxfft,
                   float2 *spec, cudaStream_t stream);

// F stage (csrc/fxb_fstage.cu).  A work item is one subband of one station
// with the one or two bands recording it; items of the same kind (FFT length,
// band packing) share a launch.
struct FGroup {
	int32_t station, freq;
	int32_t band[2];
	int32_t row[2];          // rows within the frequency's spectra (-1: band not output)
	int32_t nb;
	int32_t lsb;
	double lofreq;
	// corrections of the subband's recorded frequency (mode.cpp:870-1145,
	// 1296-1347): per band the clock term of the fractional-sample rotation,
	// fse - clk[j] (us; offset -/+ delta/2 by polarisation), and the
	// phase-offset rotation (turns); the LO offset (Hz) of the fringe rotation
	double clk[2];
	double looff;
	float phase[2];
	int32_t corr;            // any correction nonzero
	int32_t pad_;
};

#if defined(__CUDACC__)
// D (turns per channel) as hi + lo with hi holding 10 significant bits, so
// that c * hi is exact in FP32 for |c| <= 8192 and the channel phase
// c * D = (c * hi mod 1) + c * lo keeps FP32 accuracy however many turns
// c * D spans (large clock offsets)
__device__ __forceinline__ void split_turns(double D, float &hi, float &lo)
{
	int e;
	frexp(D, &e);
	const double h = D == 0.0 ? 0.0 : ldexp(rint(ldexp(D, 9 - e)), e - 9);
	hi = (float)h;
	lo = (float)(D - h);
}

// LO-offset fringe phase (turns) at wall-clock time w (seconds since the job
// start) except the per-sample term: -looff (w - int w) - frac(looff) int w,
// the integer seconds entering only through the offset's fractional part
// (mode.cpp:873-882, 932-951)
__device__ __forceinline__ double looff_wall_turns(double looff, double w)
{
	if(looff == 0.0)
		return 0.0;
	const int iw = (int)w;
	double fl = fabs(looff) - (int)fabs(looff);
	if(looff < 0)
		fl = -fl;
	return -looff * (w - iw) - (fabs(fl) > (double)1e-9f ? fl * iw : 0.0);
}
#endif

struct FKind {
	int32_t first, count;    // range of work items in the item table
	int32_t N, nb;           // FFT length, bands per item
	int32_t kb, fpc;         // radix-8 butterflies per thread and pass, FFTs side by side per CTA
	int32_t threads, tq;     // CTA size, FFT iterations per CTA
	int32_t pp, out;         // two exchange buffers (else one), output form (0 FP32 spectra, 1 tensor-core spectra)
	int32_t items_fast;      // grid order: work items fastest (else time chunks); scheduling only
	int32_t twn, tcfft;      // twiddle entries of length N; 1: tensor-core FFT kernel (fxb_fstage_tc.cu)
	size_t smem;
	const void *tw;          // twiddle table of length N (make_fstage_twiddles layout)
	const void *tctab;       // constant tables of the tensor-core FFT kernel
	const int32_t *tcpairs;  // tensor-core FFT: [tcnpairs][2] FGroup indices of each work unit's two subbands
	int32_t tcnpairs;
	int32_t tcbpt;           // tensor-core FFT: bits per time of the stations' VDIF words
	int32_t muxraw;          // 1: the items' stations hand over raw INTERLACEDVDIF reads
	int32_t cplx;            // 1: the items' stations sample complex (N = nchan points)
	int32_t persist;         // 1: run by the persistent launches (launch_fstage_multi), not launch_fstage_kind
};

// Spectra of the tensor-core forms hold X 2^-kTcSpecExp (FP16 or BF16), so
// that the largest value of any supported FFT (16384 points of 8-bit levels,
// |X| <= 16384 x 38.8) stays inside the FP16 range; the XMAC epilogue scales
// the products back by 2^(2 kTcSpecExp), exactly.
constexpr int kTcSpecExp = 5;

struct FsArgs {
	const DevStation *st;
	const DevSubintStation *sub;
	const FGroup *groups;
	const DevFreqPlan *plans;
	const uint8_t *valid;
	const uint32_t *bandok;       // per frame: bands that keep their samples (null: all)
	const uint8_t *fillok;        // per frame: no fill pattern (complex data: the window's first frame)
	int64_t valid_stride;
	const FftParam *params;
	const void *tw;          // set from FKind::tw by launch_fstage_kind
	int32_t maxN, T, tq, order;
	int32_t fraclo, pp, first, items_fast;
	void *spec;              // [t][row][chan]: float2 (out 0), or half2 / bf16x2 (out 1) scaled by 2^-kTcSpecExp
	int32_t *err;            // device error flag (bounded waits of the tensor-core FFT kernel)
	int32_t h16;             // out 1: spectra as FP16 (else BF16)
	int32_t pad_;
};

bool fstage_plan(int N, int nb, int out, FKind *k);
void launch_fstage_kind(const FKind &k, FsArgs a, cudaStream_t stream);

// The persistent F-stage launches over the CUDA-core kinds of tensor-core-
// form contexts (VDIF stations, plain or raw INTERLACEDVDIF reads) of one
// context or several: CTAs take
// work units from a list in order, each run as one CTA of launch_fstage_kind
// runs it (tq x fpc FFT times of one work item).  Narrow units (FFTs of up to
// 4096 points) run in CTAs of 256 threads, wide units (8192-point FFTs of one
// band) in CTAs of 512, one launch each.  Every tensor-core-form context runs
// these kinds this way, alone or in a batch, so results do not depend on it.
constexpr int kFsMultiMembers = 16;
constexpr int kFsMultiFc = 128;          // FFT constants of one narrow unit at most (tq x fpc)
struct FsMultiKind {
	const void *tw;                      // twiddles of length N
	int32_t member, code;                // context; 128 x raw INTERLACEDVDIF reads + 32 x bands per item + log2 N
	int32_t first, tq;                   // first FGroup of the kind, FFT iterations per unit
};
struct FsMultiUnit {
	int32_t kind, item, tchunk;
};
struct FsMultiArgs {
	FsArgs m[kFsMultiMembers];           // per context, with its subint's staging
	const FsMultiKind *kinds;
	const FsMultiUnit *units;            // six classes: wide, two-band narrow and one-band narrow units
	                                     // of plain VDIF, then of raw reads
	int32_t unit0[6], nunit[6];          // each class's first unit and units
	int32_t *ctr;                        // one counter per class, zero before the launch
};
constexpr int kFsMultiClasses = 6;
// whether a kind (FFT length N, bands per item nb) runs in the persistent
// launches, and as a wide unit; the FFT iterations per unit for a kind's tq
bool fstage_multi_shape(int N, int nb, bool *wide);
int fstage_multi_tq(int N, int nb, int tq);
cudaError_t launch_fstage_multi(const FsMultiArgs &m, int nsm, cudaStream_t stream);
// the same with the class kernels spread over streams (each kernel on the
// next stream of the set), for callers that run them as parallel branches
cudaError_t launch_fstage_multi_on(const FsMultiArgs &m, int nsm, const cudaStream_t *streams, int nstream);
// F stage of the tensor-core form with the FFT on the tensor cores (N = 2048;
// csrc/fxb_fstage_tc.cu).  Eligible: 2048-point FFTs, fringe rotation order
// 1 (or 0 with upper sidebands only), 2-bit stations of 2..32 bands (all
// stations of the kind alike), each subband's two bands in one 4-bit field,
// 16-byte aligned frames of at least 128 samples; a work unit is two
// subbands of one station with equal sideband at one FFT time.
size_t fstage_tc_tables_bytes();
void make_fstage_tc_tables(void *out);
bool fstage_tc_eligible(int N, int order, bool any_lsb);
// returns the launch's error
cudaError_t launch_fstage_tc(const FKind &k, FsArgs a, int nsm, cudaStream_t stream);

// twiddles of FFT length N, FKind::twn entries
void make_fstage_twiddles(int N, float2 *out32);

// FP32 XMAC v2 over a set of frequencies with equal (rows, channels):
// plan_idx[0..nf) index dplans.
void launch_xmac_fp32v2(const DevFreqPlan &plan0, const DevFreqPlan *dplans, const int32_t *plan_idx, int nf, int T,
                        const float2 *spec, float2 *acc, cudaStream_t stream);

// Tensor-core XMAC (csrc/fxb_xmac_tc.cu) over one group of equally shaped
// subbands whose bf16x2 spectra lie in one block [subband][Tpad][nrow][nchan].
struct TcShape {
	int32_t f8;                       // FP8 form: e4m3 pairs, K tiles of 64 times
	int32_t h16;                      // operands (or the FP8 form's source spectra) FP16, else BF16
	int32_t w8;                       // FP8 form: values per time of a block, nrow * CB padded to 8
	int32_t nrow, nchan, r2p, G, CB, Tpad;
	int32_t raw_bytes, raw_stride;    // bytes of one TMA box, stride of the raw stages
	int32_t nrs, nas;                 // raw and operand stages
	int32_t nb;                       // accumulator buffers: 2 (one CTA per SM) or 1 (two CTAs per SM)
	int32_t dstride, dump_off;        // accumulator copy: floats per row, byte offset
	size_t smem;
};
bool tc_shape(int nrow, int nchan, int T, bool f8, bool h16, TcShape *s);
// set the raw / operand ring depths and accumulator buffers of a shape (and
// its shared-memory plan); false if they do not fit (227 KB for one CTA per
// SM, 112 KB each for two)
bool tc_stages(TcShape *s, int nrs, int nas, int nb = 2);
bool tc_make_tensormap(void *map_out, const void *spec, const TcShape &s, int nf);
size_t tc_tensormap_size();
void launch_xmac_tc(const void *tmap, const TcShape &s, const DevFreqPlan *dplans, const int32_t *plan_idx, int nf,
                    int nsm, int32_t *err, float2 *acc, cudaStream_t stream);
// One launch over several groups (of one context or several) whose shapes
// share rows, form and ring depths: the CTAs stride over the groups' work
// units in turn.  Each product is added to its accumulator once per subint
// whatever the schedule, so results equal those of a launch per group.
constexpr int kXMultiGroups = 16;
struct alignas(64) TmapBytes {
	unsigned char b[128];
};
struct XGroupRec {
	const DevFreqPlan *plans;
	const int32_t *plan_idx;             // [subbands of the group] plan of each
	float2 *acc;                         // the context's accumulators
	int32_t nchan, nkt, nblk, unit0;     // channels, K tiles, channel blocks per subband, first unit
};
struct XMultiArgs {
	TmapBytes map[kXMultiGroups];        // CUtensorMap of each group's spectra block
	XGroupRec g[kXMultiGroups];
	int32_t ngroups, nunits;
};
// appends a group (false when the launch is full)
bool xmac_multi_add(XMultiArgs *xm, const void *tmap, const TcShape &s, const DevFreqPlan *dplans,
                    const int32_t *plan_idx, int nf, float2 *acc);
void launch_xmac_tc_multi(const XMultiArgs &xm, const TcShape &s, int nsm, int32_t *err, cudaStream_t stream);
// FP8 form: per subband of the group (plan_idx[nf]), the bf16x2 spectra
// [Tpad][nblk][nrow][CB] at spec_off -> e4m3x2 [Tpad][nblk][w8] at spec8_off,
// scaled per (channel, input) so that the input's largest component over the
// subint's T times maps to 240; writes 1 / scale to iscale[channel][input]
void launch_quant_fp8(const TcShape &s, const DevFreqPlan *dplans, const int32_t *plan_idx, int nf, int T,
                      const uint32_t *spec16, uint16_t *spec8, cudaStream_t stream);

// FP32 cross-multiply-accumulate of one frequency into acc.
void launch_xmac_fp32(const DevFreqPlan &plan, const DevFreqPlan *dplan, int T, const float2 *spec, float2 *acc,
                      cudaStream_t stream);

// Phase cal (csrc/fxb_pcal.cu).  A group is up to kPcalGroupBands recorded
// bands of one station with the same bin count; a band is one band's tones.
constexpr int kPcalGroupBands = 16;
struct DevPcalGroup {
	int32_t station, nb, nbins, shift;  // shift: the shifting extractor's offset (Hz), complex bins; else 0
	int64_t fs;                         // samples per second
	int32_t band[kPcalGroupBands];
	int64_t bin_off[kPcalGroupBands];   // first bin (double) of each band in the bin accumulator
};
struct DevPcalBand {
	int32_t ntones, nbins, first, step;
	int32_t shift, pad;                 // complex bins when shift != 0
	int64_t bin_off, core;
};
// shared memory of a group's lane sums (bin counts below the CTA width) and
// of one launch with tpc FFTs per chunk
size_t pcal_group_smem(const DevPcalGroup &g);
size_t pcal_smem(size_t group_smem, int tpc);
constexpr size_t kPcalSmemMax = 96 * 1024;    // lane sums of one group at most
constexpr size_t kPcalSmemLaunchMax = 200 * 1024;   // a launch's FFT table and lane sums at most
// allows the binning kernels smem bytes of dynamic shared memory (once per context)
cudaError_t pcal_init(size_t smem);
// folds the subint's samples into the FP64 bins: the FFTs are split into
// nchunk chunks, chunk c adds to bins + c * chunk_stride.  Every group of one
// launch belongs to stations of nbits-bit samples with bpt bits per time and
// to one extractor (shift: the shifting extractor's complex bins); maxbins is
// the launch's largest bin count, smem its pcal_smem.
void launch_pcal_bin(const DevPcalGroup *groups, int ngroups, int maxbins, int nchunk, int nbits, int bpt, bool shift,
                     size_t smem, const DevStation *st, const DevSubintStation *sub, const FftParam *params,
                     const uint8_t *valid, int64_t valid_stride, int T, int64_t chunk_stride, double *bins,
                     cudaStream_t stream);
// writes the tones of every band into the core result
void launch_pcal_final(const DevPcalBand *bands, int nbands, int nchunk, int64_t chunk_stride, const double *bins,
                       float2 *core, cudaStream_t stream);

// Zoom-band spectra from their parents' (after the F stage, before the
// XMAC): tc selects the tensor-core form's bf16x2 spectra.
void launch_zoom_gather(const DevZoomCopy *zc, int nzc, const DevFreqPlan *plans, int T, bool tc, void *spec,
                        cudaStream_t stream);

// pbw: per-band data weights [station][FFT][nbm] of INTERLACEDVDIF stations (null: none)
void launch_weights(const DevBWeight *bw, int nbw, const DevACWeight *acw, int nacw, const FftParam *params,
                    const float *pbw, int nbm, const DevStation *st, int T, float *bwacc, float *acwacc,
                    cudaStream_t stream);

void launch_finalise(const DevOutMap *om, int nom, int maxout, const float2 *acc, const DevBWeight *bw, int nbw,
                     const float *bwacc, const DevACWeight *acw, int nacw, const float *acwacc, float2 *core,
                     int64_t corelen, cudaStream_t stream);

void launch_vdif_unpack(const uint8_t *data, int64_t nbytes, int payload, int header, int nchan, int nbits,
                        int64_t offsetsamples, int nsamp, float *out, int *good, cudaStream_t stream);

}  // namespace fxb
