// Multi-thread VDIF to single-thread multi-channel VDIF on the device: the
// reference's VDIFMuxer (mpifxcorr/src/datamuxer.cpp:106-848), which the
// DataStream runs on every read of an INTERLACEDVDIF stream before its frames
// reach Mode.  One call takes one read: nin frames of the wanted threads
// (interleaved in any order, other threads skipped) and writes nin / nthreads
// output frames of nthreads channels each, in three launches:
//   k_mux_index    every input frame finds its place: frame slot (time since
//                  the first frame of the read, in frames) and thread
//                  (VDIFMuxer::deinterlace, datamuxer.cpp:765-846); where a
//                  slot is filled twice the later input frame wins, as the
//                  reference's in-order copy does;
//   k_mux_headers  one thread walks the output frames in order and writes
//                  their headers (VDIFMuxer::multiplex, datamuxer.cpp:680-763):
//                  complete slots take thread 0's header with one channel per
//                  thread, incomplete ones the first present thread's header
//                  marked invalid, empty ones the previous output header one
//                  frame later, marked invalid (empty slots before the first
//                  output frame are dropped);
//   k_mux_turn     corner turn of the complete slots' payloads
//                  (VDIFMuxer::cornerturn_generic, datamuxer.cpp:253-274):
//                  one CUDA thread per (output frame, input word), reading the
//                  word of every thread and writing nthreads output words.
// Byte work: HBM-bound by design (every payload byte read once, written once).

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>

#include "fxb_internal.h"
#include "fxb_kernels.h"

namespace fxb {

namespace {

constexpr int kMaxMuxThreads = 64;

struct MuxArgs {
	const uint8_t *in;
	uint8_t *out;
	int32_t *slot;                // [nslot][nthreads] input frame index or -1
	int32_t *status;              // [0] error code, [1] output frames
	int32_t tmap[kMaxMuxThreads]; // VDIF thread id of each channel
	int32_t nthreads, inframebytes, outframebytes, nin, nslot, nproc, fps, nbits;
	int32_t wordsin, spow;        // payload words per input frame, samples per output word and thread
	int32_t vec;                  // output words 16-byte aligned: vector stores
};

// VDIF header fields (vdifio.h:58-80)
__device__ __forceinline__ uint32_t hw(const uint8_t *h, int w) { return ((const uint32_t *)h)[w]; }

// MJD of the first day of a VDIF epoch (half years from 2000): days since
// 1858-11-17 of (2000 + e / 2)-(1 or 7)-01, by the civil-from-days count
__device__ __forceinline__ int epoch_mjd(int e)
{
	const int y0 = 2000 + e / 2, m = (e % 2) * 6 + 1;
	const int y = y0 - (m <= 2);
	const int era = y / 400;
	const int yoe = y - era * 400;
	const int doy = (153 * (m + (m > 2 ? -3 : 9)) + 2) / 5;
	const int doe = yoe * 365 + yoe / 4 - yoe / 100 + doy;
	return era * 146097 + doe - 678882 + 1;     // days since 0000-03-01 -> MJD
}

__device__ __forceinline__ void frame_time(const uint8_t *h, int *mjd, int *sec, int *frame)
{
	const uint32_t w0 = hw(h, 0), w1 = hw(h, 1);
	const int seconds = (int)(w0 & 0x3FFFFFFFu);
	*mjd = epoch_mjd((int)((w1 >> 24) & 0x3Fu)) + seconds / 86400;
	*sec = seconds % 86400;
	*frame = (int)(w1 & 0xFFFFFFu);
}

__global__ void k_mux_index(const MuxArgs a)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if(i >= a.nin)
		return;
	const uint8_t *h = a.in + (int64_t)i * a.inframebytes;
	const int tid = (int)((hw(h, 3) >> 16) & 0x3FFu);
	const int fbytes = (int)(hw(h, 2) & 0xFFFFFFu) * 8;
	if(fbytes != a.inframebytes)
	{
		atomicCAS(a.status, 0, 1);             // frame size changed: the reference aborts
		return;
	}
	int ti = -1;
	for(int j = 0; j < a.nthreads; j++)
		if(a.tmap[j] == tid)
		{
			ti = j;
			break;
		}
	if(ti < 0)
		return;                                 // a thread nobody asked for
	int m0, s0, f0, m, s, f;
	frame_time(a.in, &m0, &s0, &f0);
	frame_time(h, &m, &s, &f);
	const int64_t cur = ((int64_t)(m - m0) * 86400 + s - s0) * a.fps + f - f0;
	if(cur < 0)
		return;                                 // earlier than the read's first frame
	if(cur >= a.nslot)
	{
		atomicCAS(a.status, 0, 2);             // beyond the buffer: the reference aborts
		return;
	}
	atomicMax(a.slot + cur * a.nthreads + ti, i);
}

__device__ __forceinline__ void put_header(uint32_t *o, const uint32_t *src)
{
	for(int w = 0; w < 8; w++)
		o[w] = src[w];
}

// first slot holding any frame (output frames before it are dropped)
__global__ void k_mux_first(const MuxArgs a)
{
	const int k = blockIdx.x * blockDim.x + threadIdx.x;
	if(k >= a.nproc || *a.status != 0)
		return;
	const int32_t *sl = a.slot + (int64_t)k * a.nthreads;
	for(int j = 0; j < a.nthreads; j++)
		if(sl[j] >= 0)
		{
			atomicMin(a.status + 2, k);
			return;
		}
}

// the header slot k's output frame starts from, before the empty-slot step:
// complete -> thread 0's, incomplete -> the first present thread's
__device__ __forceinline__ void slot_header(const MuxArgs &a, int k, int logch, uint32_t *o, bool *all_out,
                                            bool *any_out)
{
	const int32_t *sl = a.slot + (int64_t)k * a.nthreads;
	bool all = true;
	int first = -1;
	for(int j = 0; j < a.nthreads; j++)
	{
		if(sl[j] < 0)
			all = false;
		else if(first < 0)
			first = j;
	}
	*all_out = all;
	*any_out = first >= 0;
	if(first < 0)
		return;
	put_header(o, (const uint32_t *)(a.in + (int64_t)sl[all ? 0 : first] * a.inframebytes));
	o[0] = (o[0] & 0x7FFFFFFFu) | (all ? 0u : 0x80000000u);                       // invalid
	if(all)
		o[2] = (o[2] & ~(0x1Fu << 24)) | ((uint32_t)logch << 24);             // channels
	o[2] = (o[2] & ~0xFFFFFFu) | ((uint32_t)(a.outframebytes / 8) & 0xFFFFFFu);   // frame bytes
	o[3] &= ~(0x3FFu << 16);                                                  // thread 0
}

// one thread per slot k from the first filled one: output frame k - first.
// An empty slot takes the nearest earlier filled slot's header advanced one
// frame per slot between them (the reference increments the preceding output
// header, itself such a copy), invalid; outidx[k] = output frame to corner
// turn, or -1
__global__ void k_mux_headers(const MuxArgs a, int32_t *outidx)
{
	const int k = blockIdx.x * blockDim.x + threadIdx.x;
	if(k >= a.nproc || *a.status != 0)
		return;
	const int k0 = a.status[2];
	outidx[k] = -1;
	if(k < k0)
		return;
	int logch = 0;                              // vdifio setVDIFNumChannels: floor(log2)
	for(int n = a.nthreads; n > 1; n /= 2)
		logch++;
	uint32_t *o = (uint32_t *)(a.out + (int64_t)(k - k0) * a.outframebytes);
	uint32_t h[8];
	bool all, any;
	slot_header(a, k, logch, h, &all, &any);
	if(!any)
	{
		int g = k - 1;
		bool ga = false, gy = false;
		while(true)
		{
			slot_header(a, g, logch, h, &ga, &gy);
			if(gy)
				break;
			g--;
		}
		h[0] |= 0x80000000u;
		uint32_t fr = h[1] & 0xFFFFFFu;
		uint32_t secs = h[0] & 0x3FFFFFFFu;
		for(int step = 0; step < k - g; step++)
		{
			fr = (fr + 1u) & 0xFFFFFFu;
			if((int)fr == a.fps)
			{
				fr = 0u;
				secs = (secs + 1u) & 0x3FFFFFFFu;      // vdifio setVDIFFrameSecond(second + 1)
			}
		}
		h[0] = (h[0] & 0xC0000000u) | secs;
		h[1] = (h[1] & ~0xFFFFFFu) | fr;
	}
	put_header(o, h);
	if(all)
		outidx[k] = k - k0;
	else
		for(int w = 8; w < a.outframebytes / 4; w++)
			o[w] = 0u;
	if(k == a.nproc - 1)
		a.status[1] = a.nproc - k0;
}

// corner turn: x = input word, y = slot; output word (i nthreads + j) of the
// slot's output frame packs, for k < spow and thread l, sample j spow + k of
// thread l at bit (k nthreads + l) nbits
// NT > 0: nthreads known at compile time (the words stay in registers);
// NT = 0: any count up to kMaxMuxThreads
template <int NT>
__global__ void k_mux_turn(const MuxArgs a, const int32_t *outidx)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	const int k = blockIdx.y;
	if(i >= a.wordsin || *a.status != 0)
		return;
	const int o = outidx[k];
	if(o < 0)
		return;
	const int nt = NT > 0 ? NT : a.nthreads;
	const int32_t *sl = a.slot + (int64_t)k * nt;
	uint32_t w[NT > 0 ? NT : kMaxMuxThreads];
#pragma unroll
	for(int l = 0; l < nt; l++)
		w[l] = __ldg((const uint32_t *)(a.in + (int64_t)sl[l] * a.inframebytes + 32) + i);
	const uint32_t mask = (1u << a.nbits) - 1u;
	uint32_t *dst = (uint32_t *)(a.out + (int64_t)o * a.outframebytes + 32) + (int64_t)i * nt;
	if constexpr(NT >= 4)
	{
		// NT words per input word: 16-byte stores (frames start 16-byte aligned
		// when the payload is a multiple of 16 bytes, checked on the host)
#pragma unroll
		for(int j0 = 0; j0 < NT; j0 += 4)
		{
			uint32_t v[4];
#pragma unroll
			for(int q = 0; q < 4; q++)
			{
				uint32_t word = 0u;
				for(int kk = 0; kk < a.spow; kk++)
#pragma unroll
					for(int l = 0; l < NT; l++)
						word |= ((w[l] >> (((j0 + q) * a.spow + kk) * a.nbits)) & mask) << ((kk * NT + l) * a.nbits);
				v[q] = word;
			}
			if(a.vec)
				*(uint4 *)(dst + j0) = make_uint4(v[0], v[1], v[2], v[3]);
			else
				for(int q = 0; q < 4; q++)
					dst[j0 + q] = v[q];
		}
	}
	else
	{
#pragma unroll
		for(int j = 0; j < nt; j++)
		{
			uint32_t word = 0u;
			for(int kk = 0; kk < a.spow; kk++)
#pragma unroll
				for(int l = 0; l < nt; l++)
					word |= ((w[l] >> ((j * a.spow + kk) * a.nbits)) & mask) << ((kk * nt + l) * a.nbits);
			dst[j] = word;
		}
	}
}

// ---------------------------------------------------------------- raw reads inside a context
// The same placement and headers for the stations of a context whose buffers
// are raw reads (DevStation::muxraw), without the corner turn: the F stage
// reads each band's samples from its thread's frame through the slot table.
// Grids are (work, station); stations without raw reads return at once.

__global__ void k_mr_init(const DevStation *__restrict__ st, DevSubintStation *__restrict__ sub)
{
	const int s = blockIdx.y;
	if(!st[s].muxraw)
		return;
	DevSubintStation &U = sub[s];
	const int64_t n = (int64_t)U.mux_nslot * st[s].nthr;
	for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
		U.mux_slot[i] = -1;
	if(blockIdx.x == 0 && threadIdx.x == 0)
	{
		U.mux_status[0] = 0;
		U.mux_status[1] = 0;
		U.mux_status[2] = U.mux_nproc;
	}
}

// VDIFMuxer::deinterlace (datamuxer.cpp:765-846): every input frame finds its
// slot (frames since the read's first frame) and thread; the later input
// frame wins a slot filled twice
__global__ void k_mr_index(const DevStation *__restrict__ st, DevSubintStation *__restrict__ sub)
{
	const int s = blockIdx.y;
	const DevStation &S = st[s];
	if(!S.muxraw)
		return;
	DevSubintStation &U = sub[s];
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < U.mux_nin; i += gridDim.x * blockDim.x)
	{
		const uint8_t *h = U.buf + (int64_t)i * S.inframebytes;
		const int tid = (int)((hw(h, 3) >> 16) & 0x3FFu);
		const int fbytes = (int)(hw(h, 2) & 0xFFFFFFu) * 8;
		if(fbytes != S.inframebytes)
		{
			atomicCAS(U.mux_status, 0, 1);     // frame size changed
			continue;
		}
		int ti = -1;
		for(int j = 0; j < S.nthr; j++)
			if(S.tmap[j] == tid)
			{
				ti = j;
				break;
			}
		if(ti < 0)
			continue;
		int m0, s0, f0, m, sc, f;
		frame_time(U.buf, &m0, &s0, &f0);
		frame_time(h, &m, &sc, &f);
		const int64_t cur = ((int64_t)(m - m0) * 86400 + sc - s0) * S.fps + f - f0;
		if(cur < 0)
			continue;
		if(cur >= U.mux_nslot)
		{
			atomicCAS(U.mux_status, 0, 2);     // beyond the muxer's buffer
			continue;
		}
		atomicMax(U.mux_slot + cur * S.nthr + ti, i);
	}
}

__global__ void k_mr_first(const DevStation *__restrict__ st, DevSubintStation *__restrict__ sub)
{
	const int s = blockIdx.y;
	const DevStation &S = st[s];
	if(!S.muxraw)
		return;
	DevSubintStation &U = sub[s];
	if(U.mux_status[0] != 0)
		return;
	for(int k = blockIdx.x * blockDim.x + threadIdx.x; k < U.mux_nproc; k += gridDim.x * blockDim.x)
	{
		const int32_t *sl = U.mux_slot + (int64_t)k * S.nthr;
		for(int j = 0; j < S.nthr; j++)
			if(sl[j] >= 0)
			{
				atomicMin(U.mux_status + 2, k);
				break;
			}
	}
}

// muxed payload word q of a complete slot (the corner turn of
// VDIFMuxer::cornerturn_generic, datamuxer.cpp:253-274: output word
// i nthreads + j packs, for k < spow and thread l, sample j spow + k of
// thread l at bit (k nthreads + l) nbits)
__device__ uint32_t mr_word(const DevStation &S, const DevSubintStation &U, const int32_t *sl, int q)
{
	const int nt = S.nthr, i = q / nt, j = q - i * nt;
	const int wordsin = (S.inframebytes - 32) / 4;
	const int spow = (32 / S.nbits) / nt;
	const uint32_t mask = (1u << S.nbits) - 1u;
	uint32_t word = 0u;
	for(int l = 0; l < nt; l++)
	{
		const uint32_t w = (i < wordsin) ? ((const uint32_t *)(U.buf + (int64_t)sl[l] * S.inframebytes + 32))[i] : 0u;
		for(int kk = 0; kk < spow; kk++)
			word |= ((w >> ((j * spow + kk) * S.nbits)) & mask) << ((kk * nt + l) * S.nbits);
	}
	return word;
}

// header of slot k before the empty-slot step (as slot_header above)
__device__ void mr_slot_header(const DevStation &S, const DevSubintStation &U, int k, uint32_t *o, bool *all_out,
                               bool *any_out)
{
	const int32_t *sl = U.mux_slot + (int64_t)k * S.nthr;
	bool all = true;
	int first = -1;
	for(int j = 0; j < S.nthr; j++)
	{
		if(sl[j] < 0)
			all = false;
		else if(first < 0)
			first = j;
	}
	*all_out = all;
	*any_out = first >= 0;
	if(first < 0)
		return;
	put_header(o, (const uint32_t *)(U.buf + (int64_t)sl[all ? 0 : first] * S.inframebytes));
	int logch = 0;
	for(int n = S.nthr; n > 1; n /= 2)
		logch++;
	o[0] = (o[0] & 0x7FFFFFFFu) | (all ? 0u : 0x80000000u);
	if(all)
		o[2] = (o[2] & ~(0x1Fu << 24)) | ((uint32_t)logch << 24);
	o[2] = (o[2] & ~0xFFFFFFu) | ((uint32_t)(S.framebytes / 8) & 0xFFFFFFu);
	o[3] &= ~(0x3FFu << 16);
}

// header and first / last payload words of output frame k - k0 (slot k)
__device__ void mr_header(const DevStation &S, const DevSubintStation &U, int k, int k0)
{
	uint32_t h[8];
	bool all, any;
	mr_slot_header(S, U, k, h, &all, &any);
	if(!any)
	{
		int g = k - 1;
		bool ga = false, gy = false;
		while(true)
		{
			mr_slot_header(S, U, g, h, &ga, &gy);
			if(gy)
				break;
			g--;
		}
		h[0] |= 0x80000000u;
		uint32_t fr = h[1] & 0xFFFFFFu;
		uint32_t secs = h[0] & 0x3FFFFFFFu;
		for(int step = 0; step < k - g; step++)
		{
			fr = (fr + 1u) & 0xFFFFFFu;
			if((int)fr == S.fps)
			{
				fr = 0u;
				secs = (secs + 1u) & 0x3FFFFFFFu;
			}
		}
		h[0] = (h[0] & 0xC0000000u) | secs;
		h[1] = (h[1] & ~0xFFFFFFu) | fr;
	}
	uint32_t *o = U.mux_hdr + (int64_t)(k - k0) * 16;
	put_header(o, h);
	const int words = S.payload / 4;
	const int32_t *sl = U.mux_slot + (int64_t)k * S.nthr;
	o[8] = all ? mr_word(S, U, sl, 0) : 0u;
	o[9] = all ? mr_word(S, U, sl, 1) : 0u;
	o[10] = all ? mr_word(S, U, sl, words - 2) : 0u;
	o[11] = all ? mr_word(S, U, sl, words - 1) : 0u;
}

// VDIFMuxer::multiplex headers (datamuxer.cpp:680-763) of output frame
// k - k0 for slot k, with the muxed payload's first and last 64-bit words of
// complete slots (what the frame-validity check reads)
__global__ void k_mr_headers(const DevStation *__restrict__ st, DevSubintStation *__restrict__ sub)
{
	const int s = blockIdx.y;
	const DevStation &S = st[s];
	if(!S.muxraw)
		return;
	const DevSubintStation &U = sub[s];
	if(U.mux_status[0] != 0)
		return;
	const int k0 = U.mux_status[2];
	for(int k = k0 + blockIdx.x * blockDim.x + threadIdx.x; k < U.mux_nproc; k += gridDim.x * blockDim.x)
		mr_header(S, U, k, k0);
}


// the muxed stream's length and start: leading empty slots are dropped, so
// the stream starts k0 frames after the read's first frame
__global__ void k_mr_fix(const DevStation *__restrict__ st, DevSubintStation *__restrict__ sub, int S)
{
	const int s = blockIdx.x * blockDim.x + threadIdx.x;
	if(s >= S || !st[s].muxraw)
		return;
	DevSubintStation &U = sub[s];
	if(U.mux_status[0] != 0)
	{
		U.nbytes = 0;                            // the reference aborts on such a read
		U.mux_k0 = 0;
		return;
	}
	const int k0 = U.mux_status[2];
	U.mux_k0 = k0;
	U.nbytes = (int64_t)(U.mux_nproc - k0) * st[s].framebytes;
	const int64_t ns = (int64_t)U.datans + ((int64_t)k0 * 1000000000LL) / st[s].fps;
	U.datasec += (int32_t)(ns / 1000000000LL);
	U.datans = (int32_t)(ns % 1000000000LL);
}

}  // namespace

void launch_mux_raw(const DevStation *st, DevSubintStation *sub, int S, int maxslots, int maxproc,
                    cudaStream_t stream)
{
	// fixed grids (grid-stride loops), so that a captured graph fits any read
	(void)maxslots;
	(void)maxproc;
	const dim3 g(32, S);
	k_mr_init<<<g, 256, 0, stream>>>(st, sub);
	k_mr_index<<<g, 256, 0, stream>>>(st, sub);
	k_mr_first<<<g, 256, 0, stream>>>(st, sub);
	k_mr_headers<<<g, 128, 0, stream>>>(st, sub);
	k_mr_fix<<<(S + 63) / 64, 64, 0, stream>>>(st, sub, S);
}

fxb_status vdif_mux(const uint8_t *dev_in, int64_t inbytes, int32_t nthreads, const int32_t *thread_ids,
                    int32_t inframebytes, int32_t fps, int32_t nbits, uint8_t *dev_out, int64_t outcap,
                    int64_t *outbytes, void *stream, std::string &err)
{
	cudaStream_t st = (cudaStream_t)stream;
	if(!dev_in || !dev_out || !thread_ids || !outbytes || nthreads < 1 || nthreads > kMaxMuxThreads ||
	   inframebytes <= 32 || (inframebytes - 32) % 4 != 0 || fps < 1 || nbits < 1 || nbits > 16 || inbytes < 0)
		return FXB_ERR_ARG;
	MuxArgs a;
	memset(&a, 0, sizeof(a));
	a.nthreads = nthreads;
	a.inframebytes = inframebytes;
	a.outframebytes = (inframebytes - 32) * nthreads + 32;
	a.nin = (int32_t)(inbytes / inframebytes);
	// threads' frame slots (numthreadbufframes = readframes x DEMUX_BUFFER_FACTOR / nthreads)
	a.nslot = a.nin * 4 / nthreads;
	a.fps = fps;
	a.nbits = nbits;
	a.wordsin = (inframebytes - 32) / 4;
	const int samplesperframe = ((inframebytes - 32) * 8) / nbits;
	const int spiw = samplesperframe / a.wordsin;
	a.spow = spiw / nthreads;
	if(a.spow == 0)
	{
		err = "too many threads or bits for one time step per 32-bit word";
		return FXB_ERR_UNSUPPORTED;
	}
	for(int j = 0; j < nthreads; j++)
		a.tmap[j] = thread_ids[j];
	a.vec = ((uintptr_t)dev_out % 16 == 0 && a.outframebytes % 16 == 0) ? 1 : 0;
	const int nproc = a.nin / nthreads;         // one read's output frames
	a.nproc = nproc;
	if((int64_t)nproc * a.outframebytes > outcap)
		return FXB_ERR_ARG;
	*outbytes = 0;
	if(a.nin == 0)
		return FXB_OK;
	int32_t *scratch = nullptr;
	const size_t nsl = (size_t)a.nslot * nthreads;
	cudaError_t e = cudaMallocAsync(&scratch, sizeof(int32_t) * (nsl + 4 + (size_t)nproc), st);
	if(e != cudaSuccess)
		return e == cudaErrorMemoryAllocation ? FXB_ERR_NOMEM : FXB_ERR_CUDA;
	a.slot = scratch;
	a.status = scratch + nsl;
	int32_t *outidx = scratch + nsl + 4;
	a.in = dev_in;
	a.out = dev_out;
	int32_t hst[2] = {0, 0};
	// status: [0] error, [1] output frames, [2] first filled slot
	const int32_t init[4] = {0, 0, nproc, 0};
	bool ok = cudaMemsetAsync(a.slot, 0xFF, sizeof(int32_t) * nsl, st) == cudaSuccess &&
	          cudaMemcpyAsync(a.status, init, sizeof(init), cudaMemcpyHostToDevice, st) == cudaSuccess;
	if(ok)
	{
		k_mux_index<<<(a.nin + 255) / 256, 256, 0, st>>>(a);
		if(nproc > 0)
		{
			k_mux_first<<<(nproc + 255) / 256, 256, 0, st>>>(a);
			k_mux_headers<<<(nproc + 127) / 128, 128, 0, st>>>(a, outidx);
			const dim3 grid((a.wordsin + 127) / 128, nproc);
			switch(nthreads)
			{
			case 1: k_mux_turn<1><<<grid, 128, 0, st>>>(a, outidx); break;
			case 2: k_mux_turn<2><<<grid, 128, 0, st>>>(a, outidx); break;
			case 4: k_mux_turn<4><<<grid, 128, 0, st>>>(a, outidx); break;
			case 8: k_mux_turn<8><<<grid, 128, 0, st>>>(a, outidx); break;
			case 16: k_mux_turn<16><<<grid, 128, 0, st>>>(a, outidx); break;
			default: k_mux_turn<0><<<grid, 128, 0, st>>>(a, outidx); break;
			}
		}
		ok = cudaGetLastError() == cudaSuccess &&
		     cudaMemcpyAsync(hst, a.status, sizeof(hst), cudaMemcpyDeviceToHost, st) == cudaSuccess &&
		     cudaStreamSynchronize(st) == cudaSuccess;
	}
	cudaFreeAsync(scratch, st);
	if(!ok)
		return FXB_ERR_CUDA;
	if(hst[0] == 1)
	{
		err = "VDIF frame size changed within the read";
		return FXB_ERR_DATA;
	}
	if(hst[0] == 2)
	{
		err = "VDIF frame time beyond the muxer's buffer (a large jump in the stream)";
		return FXB_ERR_DATA;
	}
	*outbytes = (int64_t)hst[1] * a.outframebytes;
	return FXB_OK;
}

}  // namespace fxb
