// Per-station F stage that allocates no memory.
//
// Some callers of this library cannot call cudaMalloc: a correlator process
// that has handed all of its device memory to a pre-sized pool at start-up, a
// real-time pipeline that forbids allocation after its set-up phase, or a host
// framework that owns every allocation itself.  fxb_station_fstage_noalloc
// serves them: the caller passes the station's VDIF bytes and the output
// buffers (all device memory it owns), and every intermediate -- station and
// band tables, twiddles, valid-FFT flags, per-frame validity and per-FFT delay
// parameters -- lives in one file-scope device array, g_noalloc_scratch.
//
// That array is fixed at kScratchBytes (under 1 MiB: at most 8192 FFTs per
// subint, 131072 VDIF frames per buffer, 4096 channels, 64 bands and 64
// frequency entries) and exists on every GPU that loads the library, until
// the process exits.  All calls on a device
// share it: each call overwrites everything it reads (nothing needs to start
// at zero), and calls whose work overlaps on the GPU -- two streams, or two
// host threads -- race on it and must be serialised by the caller.
//
// The device address of the array is taken once per device with
// cudaGetSymbolAddress, on the first call made with that device current; that
// first call should therefore come before any stream capture.

#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>

#include "fxb_internal.h"
#include "fxb_kernels.h"

namespace fxb {
cudaError_t upload_lut8(cudaStream_t stream);
}

using namespace fxb;

namespace {

constexpr int kNoallocMaxFft = 8192;          // FFTs per subint
constexpr int kNoallocMaxFrames = 131072;     // VDIF frames in one station buffer
constexpr int kNoallocMaxFreq = 64;

// Byte layout of the scratch array (each part 256-byte aligned).
constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kOffStation = 0;
constexpr size_t kOffSub = align256(kOffStation + sizeof(DevStation));
constexpr size_t kOffBands = align256(kOffSub + sizeof(DevSubintStation));
constexpr size_t kOffPlans = align256(kOffBands + sizeof(DevBand) * kMaxBandsPerStation);
constexpr size_t kOffTwiddle = align256(kOffPlans + sizeof(DevFreqPlan) * kNoallocMaxFreq);
constexpr size_t kOffFlags = align256(kOffTwiddle + sizeof(float2) * 8192);
constexpr size_t kOffValid = align256(kOffFlags + sizeof(int32_t) * (kNoallocMaxFft / kFlagsPerInt + 1));
constexpr size_t kOffParams = align256(kOffValid + kNoallocMaxFrames);
constexpr size_t kScratchBytes = align256(kOffParams + sizeof(FftParam) * kNoallocMaxFft);

static_assert(kScratchBytes < (1u << 20), "scratch must stay under 1 MiB");

__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_noalloc_mutex;

// Per-FFT data weight (Mode::getDataWeight) into the caller's buffer.
__global__ void k_param_weights(const FftParam *__restrict__ params, int T, float *__restrict__ out)
{
	int t = blockIdx.x * blockDim.x + threadIdx.x;
	if(t < T)
		out[t] = params[t].status == kFftOk ? params[t].weight : 0.0f;
}

void launch_param_weights(const FftParam *params, int T, float *out, cudaStream_t stream)
{
	k_param_weights<<<(T + 255) / 256, 256, 0, stream>>>(params, T, out);
}

void *g_noalloc_ptr[64] = {};          // device address of g_noalloc_scratch, per device
bool g_noalloc_lut[64] = {};

}  // namespace

extern "C" FXB_API fxb_status fxb_station_fstage_noalloc(const fxb_freq *freqs, int32_t nfreq,
                                                         const fxb_station *station, int32_t fringe_rot_order,
                                                         int64_t subint_ns, int32_t npoly, int32_t order,
                                                         double poly0_sec, int32_t interval_s, const double *coeffs,
                                                         const uint8_t *dev_vdif, int64_t nbytes, int32_t datasec,
                                                         int32_t datans, const int32_t *validflags, int32_t sec,
                                                         int32_t ns, float *dev_spectra, size_t spectra_floats,
                                                         float *dev_weights, size_t weight_floats, int32_t *nfft,
                                                         void *stream)
{
	if(!freqs || nfreq < 1 || nfreq > kNoallocMaxFreq || !station || !coeffs || !dev_vdif || nbytes <= 0 ||
	   !dev_spectra || fringe_rot_order < 0 || fringe_rot_order > 2 || npoly < 1 || npoly > kMaxPolys ||
	   order < 0 || order > kMaxPolyOrder || interval_s <= 0)
		return FXB_ERR_ARG;
	const fxb_station &st = *station;
	// INTERLACEDVDIF stations need per-band weights and EDV4 band blanking,
	// whose per-frame band masks do not fit the fixed scratch array
	if(st.mux_threads != 0 || st.complex_sampling != 0)
		return FXB_ERR_UNSUPPORTED;
	// per-band clock, phase and LO offsets are applied by the context path's
	// F stages only
	{
		const double *corr[4] = {st.band_clock_us, st.band_clock_delta_us, st.band_phase_deg, st.band_lo_offset_hz};
		for(int q = 0; q < 4; q++)
			for(int b = 0; corr[q] && b < st.nband && b < kMaxBandsPerStation; b++)
				if(corr[q][b] != 0.0)
					return FXB_ERR_UNSUPPORTED;
	}
	if(st.nband < 1 || st.nband > kMaxBandsPerStation || !st.band_freq || (st.nband & (st.nband - 1)) ||
	   (st.nbits != 2 && st.nbits != 8) || (st.nbits == 8 && st.nband > 4) || st.payload_bytes <= 0 ||
	   st.payload_bytes % 8 || ((int64_t)st.payload_bytes * 8) % (st.nbits * st.nband) ||
	   (st.header_bytes != 32 && st.header_bytes != 16))
		return FXB_ERR_ARG;
	for(int b = 0; b < st.nband; b++)
		if(st.band_freq[b] < 0 || st.band_freq[b] >= nfreq)
			return FXB_ERR_ARG;
	const fxb_freq &f0 = freqs[st.band_freq[0]];
	for(int b = 1; b < st.nband; b++)
		if(freqs[st.band_freq[b]].nchan != f0.nchan || freqs[st.band_freq[b]].bw_mhz != f0.bw_mhz)
			return FXB_ERR_ARG;
	if(f0.nchan < 16 || f0.nchan > 4096 || (f0.nchan & (f0.nchan - 1)) || !(f0.bw_mhz > 0.0))
		return FXB_ERR_UNSUPPORTED;
	const double fftns = 2.0 * f0.nchan * 1000.0 / (2.0 * f0.bw_mhz);
	const double bpsd = (double)subint_ns / fftns;
	const int T = (int)(bpsd + 0.5);
	if(T < 1 || std::fabs(bpsd - T) > 1e-9)
		return FXB_ERR_ARG;
	// sizes beyond the scratch array are refused, never truncated
	const int64_t framebytes = st.payload_bytes + st.header_bytes;
	const int64_t valid_stride = nbytes / st.payload_bytes + 2;
	if(T > kNoallocMaxFft || valid_stride > kNoallocMaxFrames)
		return FXB_ERR_UNSUPPORTED;
	(void)framebytes;
	if(nfft)
		*nfft = T;
	// the caller's buffers must hold the whole result: spectra [T][nband][nchan] complex, weights [T]
	if(spectra_floats < (size_t)T * st.nband * f0.nchan * 2 || (dev_weights && weight_floats < (size_t)T))
		return FXB_ERR_ARG;

	cudaStream_t cs = (cudaStream_t)stream;
	int dev = 0;
	if(cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
		return FXB_ERR_CUDA;
	unsigned char *scratch = nullptr;
	{
		std::lock_guard<std::mutex> lk(g_noalloc_mutex);
		if(!g_noalloc_ptr[dev])
		{
			void *p = nullptr;
			if(cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p)
				return FXB_ERR_CUDA;
			g_noalloc_ptr[dev] = p;
		}
		scratch = (unsigned char *)g_noalloc_ptr[dev];
		if(!g_noalloc_lut[dev])
		{
			if(upload_lut8(cs) != cudaSuccess)
				return FXB_ERR_CUDA;
			g_noalloc_lut[dev] = true;
		}
	}

	// host images of the tables (pageable: cudaMemcpyAsync consumes them before returning)
	DevStation hst;
	memset(&hst, 0, sizeof(hst));
	hst.nbits = st.nbits;
	hst.payload = st.payload_bytes;
	hst.header = st.header_bytes;
	hst.nband = st.nband;
	hst.framebytes = st.payload_bytes + st.header_bytes;
	hst.framesamples = st.payload_bytes * 8 / (st.nbits * st.nband);
	hst.gran = 8 / (st.nband * st.nbits);
	if(hst.gran <= 0) hst.gran = 1;
	hst.nchan = f0.nchan;
	hst.fftchannels = 2 * f0.nchan;
	hst.asl = calcstridelength((unsigned)f0.nchan);
	hst.sticky = (st.nbits == 8 && (st.nband == 2 || st.nband == 4)) ? 1 : 0;
	hst.bpbn = (st.nband * st.nbits) / 8;
	hst.bpbd = 1;
	if(hst.bpbn == 0)
	{
		hst.bpbn = 1;
		hst.bpbd = 8 / (st.nband * st.nbits);
	}
	hst.bw = f0.bw_mhz;
	hst.sampletime = 1.0 / (2.0 * f0.bw_mhz);
	hst.npoly = npoly;
	hst.order = order;
	hst.interval = interval_s;
	hst.poly0 = poly0_sec;
	memcpy(hst.coeffs, coeffs, sizeof(double) * npoly * (order + 1));

	DevSubintStation hsub;
	memset(&hsub, 0, sizeof(hsub));
	hsub.buf = dev_vdif;
	hsub.nbytes = nbytes;
	hsub.datasec = datasec;
	hsub.datans = datans;
	hsub.subsec = sec;
	hsub.subns = ns;

	// spectra [t][band][nchan]: every band is a row of one shared plan
	DevBand hb[kMaxBandsPerStation];
	DevFreqPlan hp[kNoallocMaxFreq];
	memset(hb, 0, sizeof(hb));
	memset(hp, 0, sizeof(hp));
	bool fraclo = false;
	for(int b = 0; b < st.nband; b++)
	{
		int f = st.band_freq[b];
		hb[b].freq = f;
		hb[b].row = b;
		hb[b].lsb = freqs[f].lower_sideband;
		hb[b].lofreq = freqs[f].freq_mhz;
		double lo = freqs[f].freq_mhz;
		if(std::fabs(lo - (int)(lo + 0.5)) > 0.000000001)
			fraclo = true;
	}
	for(int f = 0; f < nfreq; f++)
	{
		hp[f].nrow = st.nband;
		hp[f].nchan = f0.nchan;
		hp[f].spec_off = 0;
	}
	const int N = 2 * f0.nchan;
	float2 htw[4096];
	for(int k = 0; k < N / 2; k++)
	{
		double ang = -2.0 * M_PI * (double)k / (double)N;
		htw[k] = make_float2((float)cos(ang), (float)sin(ang));
	}
	const int nflagint = T / kFlagsPerInt + 1;
	int32_t hflags[kNoallocMaxFft / kFlagsPerInt + 1];
	for(int k = 0; k < nflagint; k++)
		hflags[k] = 0x3FFFFFFF;
	if(validflags)
		memcpy(hflags, validflags, sizeof(int32_t) * ((T + kFlagsPerInt - 1) / kFlagsPerInt));

	DevStation *d_st = (DevStation *)(scratch + kOffStation);
	DevSubintStation *d_sub = (DevSubintStation *)(scratch + kOffSub);
	DevBand *d_bands = (DevBand *)(scratch + kOffBands);
	DevFreqPlan *d_plans = (DevFreqPlan *)(scratch + kOffPlans);
	float2 *d_tw = (float2 *)(scratch + kOffTwiddle);
	int32_t *d_flags = (int32_t *)(scratch + kOffFlags);
	uint8_t *d_valid = (uint8_t *)(scratch + kOffValid);
	FftParam *d_params = (FftParam *)(scratch + kOffParams);

	if(cudaMemcpyAsync(d_st, &hst, sizeof(hst), cudaMemcpyHostToDevice, cs) != cudaSuccess ||
	   cudaMemcpyAsync(d_sub, &hsub, sizeof(hsub), cudaMemcpyHostToDevice, cs) != cudaSuccess ||
	   cudaMemcpyAsync(d_bands, hb, sizeof(DevBand) * st.nband, cudaMemcpyHostToDevice, cs) != cudaSuccess ||
	   cudaMemcpyAsync(d_plans, hp, sizeof(DevFreqPlan) * nfreq, cudaMemcpyHostToDevice, cs) != cudaSuccess ||
	   cudaMemcpyAsync(d_tw, htw, sizeof(float2) * (N / 2), cudaMemcpyHostToDevice, cs) != cudaSuccess ||
	   cudaMemcpyAsync(d_flags, hflags, sizeof(int32_t) * nflagint, cudaMemcpyHostToDevice, cs) != cudaSuccess)
		return FXB_ERR_CUDA;

	launch_interpolators(d_st, d_sub, 1, T, cs);
	launch_frame_valid(d_st, d_sub, d_valid, nullptr, valid_stride, 1, cs);
	launch_fft_params(d_st, d_sub, d_flags, nflagint, d_valid, nullptr, valid_stride, 1, T, fringe_rot_order,
	                  d_params, nullptr, 0, cs);
	if(launch_fstage(d_st, d_sub, d_bands, st.nband, d_plans, d_valid, valid_stride, d_params, d_tw, N, 1, T,
	                 fringe_rot_order, fraclo, N, (float2 *)dev_spectra, cs) != cudaSuccess)
		return FXB_ERR_CUDA;
	if(dev_weights)
		launch_param_weights(d_params, T, dev_weights, cs);
	if(cudaGetLastError() != cudaSuccess)
		return FXB_ERR_CUDA;
	// the host images above go out of scope on return: make sure they were consumed
	if(cudaStreamSynchronize(cs) != cudaSuccess)
		return FXB_ERR_CUDA;
	return FXB_OK;
}
