// FP64 delay model and per-FFT parameters (the K5 stage).
//
// This translation unit is compiled with --fmad=false: every double
// expression below is evaluated operation by operation with IEEE rounding,
// as the reference's C++ evaluates it, so that the integer decisions derived
// from it (nearest sample, integer delay, unpack window) are bit-identical.

#include <cuda_runtime.h>

#include "fxb_internal.h"
#include "fxb_kernels.h"

namespace fxb {

// VDIF frame validity as mark5access's unpacker sees a frame when it steps
// into it: header word 2 nonzero and invalid bit clear (format_vdif.c:
// 4009-4056), no fill pattern in the first or last 64-bit payload word
// (blanker_mark5.c:282-313).  Frames that do not fit in the buffer are
// treated as invalid.
//
// bandok (may be null): the bands of each frame that keep their samples.  On
// INTERLACEDVDIF stations a valid frame with an EDV4 validity mask blanks
// band c when mask bit c / d is clear, d = channels / mask length, with the
// geometry read from the buffer's first frame (blank_vdif_EDV4,
// format_vdif.c:4699-4780; bit 31 of the C int shift tests mask bits 31-63,
// and a 32-channel header's "good" mask is 0).  Headers whose geometry is not
// the station's blank nothing.
__device__ __forceinline__ uint32_t edv4_bands(const DevStation &S, const DevSubintStation &U, const uint8_t *f)
{
	if(U.nbytes < 32)
		return 0xFFFFFFFFu;
	// the first frame of the (muxed) stream
	const uint8_t *f0 = S.muxraw ? (const uint8_t *)U.mux_hdr : U.buf;
	const uint32_t w2 = *(const uint32_t *)(f0 + 8), w3 = *(const uint32_t *)(f0 + 12);
	const uint32_t w4 = *(const uint32_t *)(f0 + 16);
	const int ml = (int)((w4 >> 16) & 0xFFu);
	if((w4 >> 24) != 4u || ml < 1 || ml > 64)
		return 0xFFFFFFFFu;
	const int nch = 1 << ((w2 >> 24) & 31u);
	const int flen = (int)(w2 & 0xFFFFFFu) * 8;
	const int spf = (flen - 32) * 8 / (nch * (int)(((w3 >> 26) & 31u) + 1u));
	const int d = nch / ml;
	if(d < 1 || nch != S.nband || spf != S.framesamples || flen != S.framebytes)
		return 0xFFFFFFFFu;
	const uint64_t mask = *(const uint64_t *)(f + 24);
	const uint64_t good = nch < 32 ? (uint64_t)((1u << nch) - 1u) : 0u;
	if(mask == good)
		return 0xFFFFFFFFu;
	uint32_t ok = 0u;
	for(int c = 0; c < nch; c++)
	{
		const int q = c / d;
		const bool keep = q < 31 ? ((mask >> q) & 1u) != 0 : (mask & 0xFFFFFFFF80000000ULL) != 0;
		ok |= (uint32_t)keep << c;
	}
	return ok | (nch < 32 ? ~((1u << nch) - 1u) : 0u);
}

// block bx of gx blocks of station s's frame-validity pass
__device__ __forceinline__ void frame_valid_blk(const DevStation *__restrict__ st, const DevSubintStation *sub,
                                                uint8_t *__restrict__ valid, uint32_t *__restrict__ bandok,
                                                int64_t valid_stride, uint8_t *__restrict__ fillok, int s, int bx,
                                                int gx)
{
	const DevStation &S = st[s];
	const DevSubintStation &U = sub[s];
	const int64_t nframes = U.nbytes / S.framebytes;
	const uint64_t FILL = 0x1122334411223344ULL;
	for(int64_t fr = bx * (int64_t)blockDim.x + threadIdx.x; fr < valid_stride; fr += (int64_t)gx * blockDim.x)
	{
		uint8_t v = 0, nofill = 0;
		// raw INTERLACEDVDIF reads: the muxed frame's header and first and last
		// payload words as the placement kernels wrote them
		const uint8_t *f = S.muxraw ? (const uint8_t *)(U.mux_hdr + fr * 16) : U.buf + fr * S.framebytes;
		if(fr < nframes)
		{
			uint32_t w0 = *(const uint32_t *)(f);
			uint32_t w2 = *(const uint32_t *)(f + 8);
			uint64_t first, last;
			if(S.muxraw)
			{
				first = *(const uint64_t *)(f + 32);
				last = *(const uint64_t *)(f + 40);
			}
			else
			{
				first = *(const uint64_t *)(f + S.header);
				last = *(const uint64_t *)(f + S.header + (S.payload / 8 - 1) * 8);
			}
			v = (w2 != 0) && !((w0 >> 31) & 1) && first != FILL && last != FILL;
			nofill = first != FILL && last != FILL;
		}
		valid[s * valid_stride + fr] = v;
		if(fillok)
			fillok[s * valid_stride + fr] = nofill;
		if(bandok)
			bandok[s * valid_stride + fr] = (v && S.mux) ? edv4_bands(S, U, f) : 0xFFFFFFFFu;
	}
}

__global__ void k_frame_valid(const DevStation *__restrict__ st, const DevSubintStation *__restrict__ sub,
                              uint8_t *__restrict__ valid, uint32_t *__restrict__ bandok, int64_t valid_stride,
                              uint8_t *__restrict__ fillok)
{
	frame_valid_blk(st, sub, valid, bandok, valid_stride, fillok, blockIdx.y, blockIdx.x, gridDim.x);
}

// Model::calculateDelayInterpolator, order 2 (model.cpp:229-299), with the
// time span of Mode::setOffsets (mode.cpp:1546-1549).
__device__ bool delay_interpolator(const DevStation &S, int blockspersend, int sec, int ns, double *c)
{
	double offsettime = (double)sec + ((double)ns) / 1000000000.0;
	double polyoffset = -S.poly0;
	double timespan = blockspersend * 2 * S.nchan * S.sampletime / 1e6;
	if(S.cplx)
		timespan /= 2;        // mode.cpp:1546-1547
	if(S.npoly <= 0)
		return false;
	int scansample = (int)((offsettime + polyoffset) / (double)S.interval);
	if(scansample == S.npoly && ((offsettime + polyoffset - scansample * S.interval) < 1e-6))
		scansample--;
	if(scansample < 0 || scansample >= S.npoly)
		return false;
	double dt[3];
	dt[1] = offsettime + polyoffset + timespan / 2.0 - scansample * S.interval;
	dt[0] = offsettime + polyoffset - scansample * S.interval;
	dt[2] = offsettime + polyoffset + timespan - scansample * S.interval;
	double d[3];
	const double *cf = S.coeffs + scansample * (S.order + 1);
	for(int k = 0; k < 3; k++)
	{
		double tp = 1.0, sum = 0.0;
		for(int i = 0; i <= S.order; i++)
		{
			sum += tp * cf[i];
			tp = tp * dt[k];
		}
		d[k] = sum;
	}
	c[0] = (2.0 * d[0] - 4.0 * d[1] + 2.0 * d[2]) / (blockspersend * blockspersend);
	c[1] = (-3.0 * d[0] + 4.0 * d[1] - d[2]) / blockspersend;
	c[2] = d[0];
	return true;
}

// The interpolators and the frame-validity pass of a subint as one launch
// (neither reads what the other writes): blocks x < gx check station y's
// frames, block gx computes station y's interpolator.
__global__ void k_prep(const DevStation *__restrict__ st, DevSubintStation *sub, int blockspersend,
                       uint8_t *__restrict__ valid, uint32_t *__restrict__ bandok, int64_t valid_stride,
                       uint8_t *__restrict__ fillok, int gx)
{
	const int s = blockIdx.y;
	if((int)blockIdx.x < gx)
	{
		frame_valid_blk(st, sub, valid, bandok, valid_stride, fillok, s, blockIdx.x, gx);
		return;
	}
	if(threadIdx.x != 0 || sub[s].interp_given)
		return;
	double c[3] = {0.0, 0.0, 0.0};
	const bool ok = delay_interpolator(st[s], blockspersend, sub[s].subsec, sub[s].subns, c);
	sub[s].interp[0] = c[0];
	sub[s].interp[1] = c[1];
	sub[s].interp[2] = c[2];
	sub[s].invalid_subint = ok ? 0 : 1;
}

__global__ void k_interpolators(const DevStation *__restrict__ st, DevSubintStation *__restrict__ sub, int S,
                                int blockspersend)
{
	int s = blockIdx.x * blockDim.x + threadIdx.x;
	if(s >= S || sub[s].interp_given)
		return;
	double c[3] = {0.0, 0.0, 0.0};
	bool ok = delay_interpolator(st[s], blockspersend, sub[s].subsec, sub[s].subns, c);
	sub[s].interp[0] = c[0];
	sub[s].interp[1] = c[1];
	sub[s].interp[2] = c[2];
	sub[s].invalid_subint = ok ? 0 : 1;
}

struct Nearest {
	bool inrange;
	int nearest;
	double starttime, averagedelay;
};

// mode.cpp:686-716: FFT-centre delay, nearest sample and range check.
__device__ Nearest nearest_sample(const DevStation &S, const DevSubintStation &U, int offsetsec, int offsetns, int i)
{
	Nearest r;
	const double *interp = U.interp;
	double fftcentre = i + 0.5;
	r.averagedelay = interp[0] * fftcentre * fftcentre + interp[1] * fftcentre + interp[2];
	double fftstartmicrosec = (i * S.fftchannels) * S.sampletime;
	r.starttime = (offsetsec - U.datasec) * 1000000.0 +
	              ((double)((long long)offsetns - (long long)U.datans)) / 1000.0 + fftstartmicrosec - r.averagedelay;
	r.nearest = (int)(r.starttime / S.sampletime + 0.5);
	long long lim = (((long long)(r.nearest + S.fftchannels) / 1) * S.bpbn) / S.bpbd;
	r.inrange = !(r.nearest < -1 || lim > U.nbytes);
	return r;
}

__device__ inline bool flag_valid(const int32_t *vf, int i)
{
	return ((vf[i / kFlagsPerInt] >> (i % kFlagsPerInt)) & 0x01) != 0;
}

// Per (station, FFT): Mode::process up to the fringe-rotation coefficients
// (mode.cpp:671-840) and the Mk5Mode::unpack weight (mk5mode.cpp:104-177).
__global__ void k_fft_params(const DevStation *__restrict__ st, const DevSubintStation *__restrict__ sub,
                             const int32_t *__restrict__ validflags, int nflagint, const uint8_t *__restrict__ valid,
                             const uint32_t *__restrict__ bandok, int64_t valid_stride, int T, int order,
                             FftParam *__restrict__ out, float *__restrict__ pbw, int nbm,
                             const uint8_t *__restrict__ fillok)
{
	const int s = blockIdx.y;
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if(i >= T)
		return;
	const DevStation &S = st[s];
	// per-band weights of INTERLACEDVDIF stations (Mk5Mode::unpack,
	// mk5mode.cpp:145-166): zero unless this FFT is unpacked (mode.cpp:663-668)
	float *pb = (S.mux && pbw) ? pbw + ((int64_t)s * T + i) * nbm : nullptr;
	if(pb)
		for(int b = 0; b < S.nband; b++)
			pb[b] = 0.0f;
	const DevSubintStation &U = sub[s];
	const int offsetsec = U.subsec, offsetns = U.subns;
	const int32_t *vf = validflags + (int64_t)s * nflagint;
	FftParam p;
	p.status = kFftZero;
	p.nearest = 0;
	p.stuck = 0;
	p.weight = 0.0f;
	p.fse = 0.0f;
	p.fmask = 0u;
	p.averagedelay = 0.0;
	p.a = p.b = p.c = 0.0;
	p.integerdelay = 0;
	p.mflags = 0;

	if(U.nbytes <= 1 || U.invalid_subint || !flag_valid(vf, i))
	{
		out[(int64_t)s * T + i] = p;
		return;
	}
	Nearest nr = nearest_sample(S, U, offsetsec, offsetns, i);
	if(!nr.inrange)
	{
		out[(int64_t)s * T + i] = p;
		return;
	}
	int nearest = nr.nearest;
	const int N = S.fftchannels;
	if(nearest == -1)
		nearest = 0;
	else if(i > 0 && !(U.nbytes <= 1) && flag_valid(vf, i - 1))
	{
		// Mode::process unpacks only when the FFT leaves the previous unpack
		// window (mode.cpp:717-724).  With unpacksamples == fftchannels that
		// window is the previous FFT's granule start alone.
		Nearest prev = nearest_sample(S, U, offsetsec, offsetns, i - 1);
		if(prev.inrange)
		{
			int pn = prev.nearest == -1 ? 0 : prev.nearest;
			int ups = pn - (pn % S.gran);
			if(!(nearest < ups || nearest > ups))
			{
				out[(int64_t)s * T + i] = p;
				return;
			}
		}
	}

	// Unpack window [ups, ups + samplestounpack) and good samples in it.
	const int ups = nearest - (nearest % S.gran);
	const int stu = N + (S.gran > 1 ? S.gran : 0);
	int count = 0;
	int stuck = N;
	int inv[32];                 // samples of EDV4-blanked bands in valid frames, per band
	int totinv = 0;
	if(pb)
		for(int b = 0; b < S.nband; b++)
			inv[b] = 0;
	{
		int64_t g0 = ups, g1 = (int64_t)ups + stu;            // [g0, g1)
		int64_t f0 = g0 / S.framesamples, f1 = (g1 - 1) / S.framesamples;
		bool blanked = false;
		for(int64_t fr = f0; fr <= f1; fr++)
		{
			int64_t a = fr * S.framesamples, b = a + S.framesamples;
			if(a < g0) a = g0;
			if(b > g1) b = g1;
			// complex data: the unpack's first frame is checked for fill
			// pattern only (mark5_stream_unpacker.c:189, a second blanker call)
			bool v = fr < valid_stride && ((S.cplx && fillok && fr == f0) ? fillok[(int64_t)s * valid_stride + fr] != 0
			                                                                : valid[(int64_t)s * valid_stride + fr] != 0);
			if(S.sticky && !v && !blanked)
			{
				blanked = true;
				stuck = (int)(a - nearest);
			}
			if(v && !(S.sticky && blanked))
			{
				// samples of this frame inside the FFT window [nearest, nearest+N)
				int64_t wa = a < nearest ? nearest : a;
				int64_t wb = b > (int64_t)nearest + N ? (int64_t)nearest + N : b;
				if(wb > wa)
				{
					count += (int)(wb - wa);
					const uint32_t bo = (pb && bandok) ? bandok[(int64_t)s * valid_stride + fr] : 0xFFFFFFFFu;
					if(bo != 0xFFFFFFFFu)
						for(int b = 0; b < S.nband; b++)
							if(!((bo >> b) & 1u))
							{
								inv[b] += (int)(wb - wa);
								totinv += (int)(wb - wa);
							}
				}
			}
		}
	}
	float weight = __fdiv_rn((float)count, (float)N);
	if(pb)
	{
		// float arithmetic of the reference: goodsamples - invalid[b] per band,
		// goodsamples - totalinvalid / nchan for the FFT's own weight
		const float gs = (float)count;
		for(int b = 0; b < S.nband; b++)
			pb[b] = __fdiv_rn(__fsub_rn(gs, (float)inv[b]), (float)N);
		weight = __fdiv_rn(__fsub_rn(gs, __fdiv_rn((float)totinv, (float)S.nband)), (float)N);
		if(!(weight > 0.0f))
			for(int b = 0; b < S.nband; b++)
				pb[b] = 0.0f;
	}
	if(!(weight > 0.0f))
	{
		out[(int64_t)s * T + i] = p;
		return;
	}
	p.status = kFftOk;
	p.nearest = nearest;
	p.stuck = stuck;
	{
		// frame-validity mask of the FFT window for the F stage
		const int64_t fa = nearest / S.framesamples;
		const int64_t nwf = (nearest - fa * S.framesamples + N - 1) / S.framesamples + 1;
		uint32_t m = 0u;
		for(int k = 0; k < 32 && k < nwf; k++)
		{
			const int64_t fr = fa + k;
			const bool vk = fr < valid_stride &&
			                ((S.cplx && fillok && k == 0) ? fillok[(int64_t)s * valid_stride + fr] != 0
			                                              : valid[(int64_t)s * valid_stride + fr] != 0);
			if(vk)
				m |= 1u << k;
		}
		p.fmask = m;
		p.mflags = nwf <= 32 ? 1 : 0;
	}
	p.weight = weight;
	p.fse = (float)(nr.starttime - nearest * S.sampletime);
	p.averagedelay = nr.averagedelay;
	const double *interp = U.interp;
	if(order == 0)
	{
		p.integerdelay = (int)nr.averagedelay;
	}
	else if(order == 1)
	{
		double d0 = interp[0] * i * i + interp[1] * i + interp[2];
		double d1 = interp[0] * (i + 0.5) * (i + 0.5) + interp[1] * (i + 0.5) + interp[2];
		double d2 = interp[0] * (i + 1) * (i + 1) + interp[1] * (i + 1) + interp[2];
		double a = d2 - d0;
		double b = d0 + (d1 - (a * 0.5 + d0)) / 3.0;
		p.integerdelay = (int)b;
		b -= p.integerdelay;
		p.a = a;
		p.b = b;
	}
	else
	{
		double a = interp[0];
		double b = interp[1] + i * interp[0] * 2.0;
		double c = interp[2] + i * interp[1] + (i * i) * interp[0];
		p.integerdelay = (int)c;
		c -= p.integerdelay;
		p.a = a;
		p.b = b;
		p.c = c;
	}
	out[(int64_t)s * T + i] = p;
}

void launch_frame_valid(const DevStation *st, const DevSubintStation *sub, uint8_t *valid, uint32_t *bandok,
                        int64_t valid_stride, int S, cudaStream_t stream, uint8_t *fillok)
{
	dim3 grid((unsigned)((valid_stride + 255) / 256 < 64 ? (valid_stride + 255) / 256 : 64), S);
	k_frame_valid<<<grid, 256, 0, stream>>>(st, sub, valid, bandok, valid_stride, fillok);
}

void launch_prep(const DevStation *st, DevSubintStation *sub, int S, int blockspersend, uint8_t *valid,
                 uint32_t *bandok, int64_t valid_stride, cudaStream_t stream, uint8_t *fillok)
{
	const int gx = (int)((valid_stride + 255) / 256 < 64 ? (valid_stride + 255) / 256 : 64);
	k_prep<<<dim3(gx + 1, S), 256, 0, stream>>>(st, sub, blockspersend, valid, bandok, valid_stride, fillok, gx);
}

void launch_interpolators(const DevStation *st, DevSubintStation *sub, int S, int blockspersend, cudaStream_t stream)
{
	k_interpolators<<<(S + 63) / 64, 64, 0, stream>>>(st, sub, S, blockspersend);
}

void launch_fft_params(const DevStation *st, const DevSubintStation *sub, const int32_t *validflags, int nflagint,
                       const uint8_t *valid, const uint32_t *bandok, int64_t valid_stride, int S, int T, int order,
                       FftParam *out, float *pbw, int nbm, cudaStream_t stream, const uint8_t *fillok)
{
	dim3 grid((T + 127) / 128, S);
	k_fft_params<<<grid, 128, 0, stream>>>(st, sub, validflags, nflagint, valid, bandok, valid_stride, T, order, out,
	                                       pbw, nbm, fillok);
}

}  // namespace fxb
