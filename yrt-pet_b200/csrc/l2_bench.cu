// L2 request throughput of this GPU: the ceiling of the fused EM kernel,
// whose image (42 MB at 256x256x160) stays resident in L2 while every voxel
// crossing of the back projection becomes a reduction request and every
// crossing of the forward projection a read.
//
// Each thread issues `iters * kUnroll` requests to uniformly random aligned
// groups of four floats inside L2-resident buffers (no two lanes of a warp
// share a sector, like the crossings of 32 different rays).  The buffer is
// split in two halves, like the EM kernel's two images: reads go to the
// first half, reductions to the second (modes 0 and 1 use the second only):
//   mode 0: red.global.add.f32       (one float of the group)
//   mode 1: red.global.add.v4.f32    (the whole group)
//   mode 2: ld.global.cg.f32         (L2 reads, L1 bypassed)
//   mode 3: per unit, one ld.global.cg.f32 and one red.global.add.v4.f32
//           from every thread (the 8 reads of a round are issued first)
//   mode 4: the same 1:1 mix split by warps: even warps read, odd warps
//           reduce (the EM kernel's warps are in their forward walks and in
//           their back projections at the same time)
// The host side times a launch with CUDA events; requests per launch are
// threads * iters * kUnroll (twice that for mode 3).  The values read do not
// matter, only the requests.
//
// Built into its own library (libyrtb_l2bench.so), used only by the
// benchmark's roofline; no counterpart in the reference.
#include <cstdint>
#include <cuda_runtime.h>

namespace
{
constexpr int kUnroll = 8;

// Integer hash "lowbias32" (C. Wellons, public domain): spreads the LCG
// state over the groups.
__device__ __forceinline__ uint32_t hash32(uint32_t x)
{
	x ^= x >> 16;
	x *= 0x7feb352du;
	x ^= x >> 15;
	x *= 0x846ca68bu;
	x ^= x >> 16;
	return x;
}

template <int MODE>
__global__ void __launch_bounds__(256)
    k_l2_requests(float* __restrict__ buf, uint32_t groups, int iters,
                  float* __restrict__ sink)
{
	// Reads: groups [0, groups); reductions: groups [groups, 2 groups).
	float* red = buf + 4ull * groups;
	const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
	uint32_t s = hash32(tid * 0x9e3779b9u + 1u);
	float acc = 0.f;
	// Mode 4: this warp's kind of request.
	const int kind = MODE == 4 ? ((threadIdx.x >> 5) & 1) + 1 : MODE;
	for (int i = 0; i < iters; i++)
	{
		uint32_t h[kUnroll];
#pragma unroll
		for (int u = 0; u < kUnroll; u++)
		{
			s = s * 1664525u + 1013904223u;  // LCG (Numerical Recipes constants)
			h[u] = hash32(s);
		}
		if (kind == 2 || kind == 3)
		{
			float v[kUnroll];
#pragma unroll
			for (int u = 0; u < kUnroll; u++)
				v[u] = __ldcg(buf + 4ull * __umulhi(h[u], groups) + (h[u] & 3u));
#pragma unroll
			for (int u = 0; u < kUnroll; u++)
				acc += v[u];
		}
#pragma unroll
		for (int u = 0; u < kUnroll; u++)
		{
			if (kind == 0)
			{
				float* g = red + 4ull * __umulhi(h[u], groups) + (h[u] & 3u);
				asm volatile("red.global.add.f32 [%0], %1;" ::"l"(g), "f"(1.0f));
			}
			else if (kind == 1 || kind == 3)
			{
				const uint32_t r = kind == 3 ? hash32(h[u] ^ 0x5bd1e995u) : h[u];
				float* g = red + 4ull * __umulhi(r, groups);
				asm volatile("red.global.add.v4.f32 [%0], {%1, %1, %1, %1};" ::"l"(g),
				             "f"(1.0f));
			}
		}
	}
	if (kind >= 2)
		if (acc == -1.0f)  // never true for the non-negative buffer; keeps the reads
			*sink = acc;
}
}  // namespace

extern "C" {

// Launches one measurement over buf (n floats, device memory, 16-byte
// aligned, n >= 8, contents non-negative; two halves of n/8 groups of four
// floats each) on stream; sink: one device float.
// blocks * 256 threads, each issuing iters * 8 requests (16 for mode 3).
// Returns 0, or a cudaError_t value (1000 for invalid arguments).
int yrtb_l2bench_launch(float* buf, uint64_t n, int mode, int iters,
                        unsigned blocks, float* sink, cudaStream_t stream)
{
	if (!buf || !sink || n < 8 || n / 8 > 0xffffffffull || iters <= 0 || blocks == 0 ||
	    (reinterpret_cast<uintptr_t>(buf) & 15u) != 0 || mode < 0 || mode > 4)
		return 1000;
	const uint32_t groups = static_cast<uint32_t>(n / 8);
	switch (mode)
	{
	case 0: k_l2_requests<0><<<blocks, 256, 0, stream>>>(buf, groups, iters, sink); break;
	case 1: k_l2_requests<1><<<blocks, 256, 0, stream>>>(buf, groups, iters, sink); break;
	case 2: k_l2_requests<2><<<blocks, 256, 0, stream>>>(buf, groups, iters, sink); break;
	case 3: k_l2_requests<3><<<blocks, 256, 0, stream>>>(buf, groups, iters, sink); break;
	default: k_l2_requests<4><<<blocks, 256, 0, stream>>>(buf, groups, iters, sink); break;
	}
	return static_cast<int>(cudaGetLastError());
}

// Requests one launch issues.
uint64_t yrtb_l2bench_requests(int mode, int iters, unsigned blocks)
{
	const uint64_t per = static_cast<uint64_t>(iters) * kUnroll * (mode == 3 ? 2 : 1);
	return per * blocks * 256ull;
}

}  // extern "C"
