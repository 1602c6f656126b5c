// FP32 cross-multiply-accumulate (Core::processdata, mpifxcorr/src/core.cpp:
// 877-972, with the autocorrelations of mode.cpp:1293-1369) for sm_100a.
//
// For one subband V[i][j] = sum_t X_i(t) X_j(t)^* over all input rows i, j is a
// complex Hermitian rank-T update per channel.  A CTA owns 32 channels of one
// subband and every 4x4 tile pair (ti <= tj) of the rows -- one warp per tile
// pair, one channel per lane -- so each spectrum value is read from HBM once
// and reused by every tile pair in shared memory.  The time axis streams
// through a two-stage cp.async pipeline (TC FFTs per stage).  Each (output,
// channel) accumulator is owned by one thread, which adds its subint sum.

#include <cuda_runtime.h>
#include <cstdint>

#include "fxb_internal.h"
#include "fxb_kernels.h"

namespace fxb {

namespace {

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
	unsigned s = (unsigned)__cvta_generic_to_shared(smem);
	asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;\n" ::); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::); }

constexpr int kCB = 32;   // channels per CTA

}  // namespace

__global__ void __launch_bounds__(512) k_xmac_fp32v2(const DevFreqPlan *__restrict__ plans,
                                                     const int32_t *__restrict__ plan_idx, int T, int TC,
                                                     const float2 *__restrict__ spec, float2 *__restrict__ acc)
{
	extern __shared__ __align__(16) float2 sx2[];
	const DevFreqPlan P = plans[plan_idx[blockIdx.y]];
	const int c0 = blockIdx.x * kCB;
	if(c0 >= P.nchan)
		return;
	const int nwarps = blockDim.x >> 5;
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int pairidx = blockIdx.z * nwarps + warp;
	const bool active = pairidx < P.npair;
	int ti = 0, tj = 0;
	if(active)
	{
		ti = P.pairs[2 * pairidx];
		tj = P.pairs[2 * pairidx + 1];
	}
	const int nrowpad = P.ntr * kTile;
	const int stage_elems = TC * nrowpad * kCB;
	const float2 *X = spec + P.spec_off;

	auto load_stage = [&](int buf, int tbase) {
		const int n16 = TC * nrowpad * (kCB / 2);
		for(int e = threadIdx.x; e < n16; e += blockDim.x)
		{
			const int ch2 = e % (kCB / 2);
			const int r = (e / (kCB / 2)) % nrowpad;
			const int tt = e / ((kCB / 2) * nrowpad);
			float2 *dst = sx2 + buf * stage_elems + (tt * nrowpad + r) * kCB + 2 * ch2;
			const int t = tbase + tt;
			const int c = c0 + 2 * ch2;
			if(t < T && r < P.nrow && c < P.nchan)
				cp_async16(dst, X + ((int64_t)t * P.nrow + r) * P.nchan + c);
			else
				*(float4 *)dst = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
		}
		cp_async_commit();
	};

	float vr[4][4], vi[4][4];
#pragma unroll
	for(int i = 0; i < 4; i++)
#pragma unroll
		for(int j = 0; j < 4; j++)
		{
			vr[i][j] = 0.0f;
			vi[i][j] = 0.0f;
		}

	load_stage(0, 0);
	int it = 0;
	for(int tb = 0; tb < T; tb += TC, it++)
	{
		const bool more = tb + TC < T;
		if(more)
		{
			load_stage((it + 1) & 1, tb + TC);
			cp_async_wait1();
		}
		else
			cp_async_wait0();
		__syncthreads();
		if(active)
		{
			const float2 *base = sx2 + (it & 1) * stage_elems;
			const int tcnt = min(TC, T - tb);
			for(int tt = 0; tt < tcnt; tt++)
			{
				const float2 *row = base + tt * nrowpad * kCB;
				float2 a[4], b[4];
#pragma unroll
				for(int i = 0; i < 4; i++)
				{
					a[i] = row[(ti * 4 + i) * kCB + lane];
					b[i] = row[(tj * 4 + i) * kCB + lane];
				}
#pragma unroll
				for(int i = 0; i < 4; i++)
#pragma unroll
					for(int j = 0; j < 4; j++)
					{
						vr[i][j] = fmaf(a[i].x, b[j].x, fmaf(a[i].y, b[j].y, vr[i][j]));
						vi[i][j] = fmaf(a[i].y, b[j].x, fmaf(-a[i].x, b[j].y, vi[i][j]));
					}
			}
		}
		__syncthreads();
	}
	if(!active)
		return;
	const int c = c0 + lane;
	if(c >= P.nchan)
		return;
#pragma unroll
	for(int i = 0; i < 4; i++)
#pragma unroll
		for(int j = 0; j < 4; j++)
		{
			const int ri = ti * 4 + i, rj = tj * 4 + j;
			if(ri >= P.nrow || rj >= P.nrow || (ti == tj && i > j))
				continue;
			const int dA = P.destA[ri * P.nrow + rj];
			const int dB = P.destB[ri * P.nrow + rj];
			if(dA >= 0)
			{
				float2 *d = acc + P.acc_off + (int64_t)dA * P.acc_ostride + (int64_t)c * P.acc_cstride;
				float2 o = *d;
				*d = make_float2(o.x + vr[i][j], o.y + vi[i][j]);
			}
			if(dB >= 0)
			{
				float2 *d = acc + P.acc_off + (int64_t)dB * P.acc_ostride + (int64_t)c * P.acc_cstride;
				float2 o = *d;
				*d = make_float2(o.x + vr[i][j], o.y - vi[i][j]);
			}
		}
}

void launch_xmac_fp32v2(const DevFreqPlan &plan0, const DevFreqPlan *dplans, const int32_t *plan_idx, int nf, int T,
                        const float2 *spec, float2 *acc, cudaStream_t stream)
{
	const int nrowpad = plan0.ntr * kTile;
	int TC = (48 * 1024) / (nrowpad * kCB * (int)sizeof(float2));
	if(TC > 16) TC = 16;
	if(TC < 1) TC = 1;
	const size_t smem = (size_t)2 * TC * nrowpad * kCB * sizeof(float2);
	int nwarps = plan0.npair < 16 ? plan0.npair : 16;
	const int zsplit = (plan0.npair + nwarps - 1) / nwarps;
	cudaFuncSetAttribute(k_xmac_fp32v2, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024);
	dim3 grid((plan0.nchan + kCB - 1) / kCB, nf, zsplit);
	k_xmac_fp32v2<<<grid, 32 * nwarps, smem, stream>>>(dplans, plan_idx, T, TC, spec, acc);
}

}  // namespace fxb
