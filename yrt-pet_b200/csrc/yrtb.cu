// libyrtb: B200 (sm_100a) kernels and C ABI for YRT-PET's projection path.
//
// Layout in HBM
//   events   structure-of-arrays, one entry per event (detector ids u32 x2,
//            TOF f32, frame i32, correction factors f32), device resident
//            across OSEM iterations; subsets are index ranges.
//   LUT      crystal centres and orientations as float4 pairs (32 B per
//            crystal, L2 resident: 1.7 MB for 53,760 crystals).
//   images   float32 [t][z][y][x]; forward projection gathers from them,
//            back projection scatters with fire-and-forget float reductions
//            (red.global.add.f32) that resolve in L2 (the 4-42 MB images of
//            the target workloads stay L2 resident on B200's 126 MB L2).
//            Deterministic projectors scatter into a 64-bit fixed-point
//            image instead (integer addition is associative, so the result
//            does not depend on the order in which the reductions land).
//
// Projection kernels run one event (or histogram bin) per thread, or per
// group of 2-4 threads that split the ray: every voxel crossing is an
// independent L2 transaction, no inter-thread synchronisation is needed, and
// the threads of a warp stay converged (events are ordered by ray length
// beforehand).  Image-space kernels are grid-stride loops sized to a multiple
// of the SM count.

#include "yrt_b200.h"
#include "device.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

using namespace yrtb;

namespace
{
thread_local std::string g_lastError;

yrtb_status fail(yrtb_status code, const std::string& msg)
{
	g_lastError = msg;
	return code;
}

#define YRTB_CUDA(call)                                                      \
	do                                                                       \
	{                                                                        \
		cudaError_t e_ = (call);                                             \
		if (e_ != cudaSuccess)                                               \
			return fail(YRTB_ERR_CUDA, std::string(#call) + ": " +           \
			                               cudaGetErrorString(e_));          \
	} while (0)

#define YRTB_LAUNCHED()                                                      \
	do                                                                       \
	{                                                                        \
		cudaError_t e_ = cudaGetLastError();                                 \
		if (e_ != cudaSuccess)                                               \
			return fail(YRTB_ERR_CUDA,                                       \
			            std::string("kernel launch: ") + cudaGetErrorString(e_)); \
	} while (0)

constexpr int kBlock = 256;

// ------------------------------------------------------ Histogram3D maps --
// Integer maps of the reference Histogram3D (Histogram3D.cpp:165-450) in a
// form a kernel can evaluate: the in-ring pair <-> (r, phi) map becomes a
// dense dpr x dpr table, the z-bin decode loop becomes a table of (z1, z2).
struct H3Host
{
	uint64_t numR, numPhi, numZBin, numZBinDiff, numDOIPoss, rCut;
	uint64_t dpr, rings, ndoi, mrd;
	std::vector<int32_t> ringMap;  // d1_ring*dpr + d2_ring -> r_ring*dpr + phi | -1
	std::vector<int2> zPairs;      // z_bin -> (z1, z2)

	void pairInRing(uint64_t r_ring, uint64_t phi, uint32_t& a, uint32_t& b) const
	{
		const int n = static_cast<int>(dpr);
		const int r = static_cast<int>(r_ring);
		const int d02 = (phi % 2 != 0) ? n / 2 + 1 : n / 2;
		int dr1 = r - n / 4 + static_cast<int>(rCut);
		int dr2 = d02 - (r - n / 4 + static_cast<int>(rCut));
		if (dr1 < 0)
			dr1 += n;
		if (dr2 < 0)
			dr2 += n;
		a = static_cast<uint32_t>((dr1 + static_cast<int>(phi) / 2) % n);
		b = static_cast<uint32_t>((dr2 + static_cast<int>(phi) / 2) % n);
		if (a > b)
			std::swap(a, b);
	}

	explicit H3Host(const yrtb_scanner& s)
	{
		dpr = s.dets_per_ring;
		rings = s.num_rings;
		ndoi = s.num_doi;
		mrd = s.max_ring_diff;
		rCut = s.min_ang_diff / 2;
		if (s.min_ang_diff % 2 != 0 && dpr % 4 == 0)
			rCut++;
		numDOIPoss = ndoi * ndoi;
		numR = numDOIPoss * (dpr / 2 + 1 - s.min_ang_diff);
		numPhi = dpr;
		const uint64_t nz = (mrd + 1) * rings - (mrd * (mrd + 1)) / 2;
		numZBinDiff = nz - rings;
		numZBin = nz + numZBinDiff;
		ringMap.assign(dpr * dpr, -1);
		for (uint64_t phi = 0; phi < numPhi; phi++)
			for (uint64_t r = 0; r < numR / numDOIPoss; r++)
			{
				uint32_t a, b;
				pairInRing(r, phi, a, b);
				ringMap[a * dpr + b] = static_cast<int32_t>(r * dpr + phi);
			}
		zPairs.resize(numZBin);
		for (uint64_t zb = 0; zb < numZBin; zb++)
		{
			int z1, z2;
			if (zb < rings)
			{
				z1 = z2 = static_cast<int>(zb);
			}
			else
			{
				int cur = (static_cast<int>(zb) - static_cast<int>(rings)) %
				              static_cast<int>(numZBinDiff) +
				          static_cast<int>(rings);
				int planes = static_cast<int>(rings);
				int dz = 0;
				while (cur - planes >= 0)
				{
					cur -= planes;
					planes -= 1;
					dz++;
				}
				z1 = cur;
				z2 = z1 + dz;
				if (zb - rings >= numZBinDiff)
					std::swap(z1, z2);
			}
			zPairs[zb] = make_int2(z1, z2);
		}
	}
};

struct H3Dev
{
	uint32_t numDets;
	const int32_t* ringMap;
	const int2* zPairs;
	uint32_t dpr, rings, ndoi, numDOIPoss, rCut;
	uint32_t mrd;
	uint64_t numR, numPhi, numZBin, numZBinDiff;
};

__device__ __forceinline__ bool h3Bin(const H3Dev& h, uint32_t d1, uint32_t d2,
                                      uint64_t& out)
{
	if ((d1 == 0 && d2 == 0) || d1 >= h.numDets || d2 >= h.numDets)
		return false;
	if (d1 > d2)
	{
		const uint32_t t = d1;
		d1 = d2;
		d2 = t;
	}
	uint32_t r1 = d1 % h.dpr, r2 = d2 % h.dpr;
	if (r1 > r2)
	{
		uint32_t t = d1;
		d1 = d2;
		d2 = t;
		t = r1;
		r1 = r2;
		r2 = t;
	}
	const int32_t m = __ldg(h.ringMap + static_cast<uint64_t>(r1) * h.dpr + r2);
	if (m < 0)
		return false;
	const uint64_t r_ring = static_cast<uint32_t>(m) / h.dpr;
	const uint64_t phi = static_cast<uint32_t>(m) % h.dpr;
	const uint64_t ringDets = static_cast<uint64_t>(h.rings) * h.dpr;
	const uint64_t doi1 = d1 / ringDets, doi2 = d2 / ringDets;
	const uint64_t r = r_ring * h.numDOIPoss + (doi1 + doi2 * h.ndoi);
	const int z1 = static_cast<int>((d1 / h.dpr) % h.rings);
	const int z2 = static_cast<int>((d2 / h.dpr) % h.rings);
	const uint32_t dz = static_cast<uint32_t>(abs(z2 - z1));
	if (dz > h.mrd)
		return false;
	const uint64_t removed = static_cast<uint64_t>(dz) * (dz - 1) / 2;
	uint64_t zb = static_cast<uint64_t>(dz) * h.rings + min(z1, z2) - removed;
	if (dz > 0 && z1 > z2)
		zb += h.numZBinDiff;
	out = zb * h.numPhi * h.numR + phi * h.numR + r;
	return true;
}

__device__ __forceinline__ void h3Pair(const H3Dev& h, uint64_t bin,
                                       uint32_t& d1, uint32_t& d2)
{
	const uint64_t z_bin = bin / (h.numPhi * h.numR);
	const uint64_t rem = bin % (h.numPhi * h.numR);
	const uint32_t phi = static_cast<uint32_t>(rem / h.numR);
	const uint32_t r = static_cast<uint32_t>(rem % h.numR);
	const int n = static_cast<int>(h.dpr);
	const int rr = static_cast<int>(r / h.numDOIPoss);
	const int d02 = (phi % 2 != 0) ? n / 2 + 1 : n / 2;
	int dr1 = rr - n / 4 + static_cast<int>(h.rCut);
	int dr2 = d02 - (rr - n / 4 + static_cast<int>(h.rCut));
	if (dr1 < 0)
		dr1 += n;
	if (dr2 < 0)
		dr2 += n;
	uint32_t a = static_cast<uint32_t>((dr1 + static_cast<int>(phi) / 2) % n);
	uint32_t b = static_cast<uint32_t>((dr2 + static_cast<int>(phi) / 2) % n);
	if (a > b)
	{
		const uint32_t t = a;
		a = b;
		b = t;
	}
	if (a == b)
	{
		d1 = d2 = 0;
		return;
	}
	const uint32_t doi_case = r % h.numDOIPoss;
	const uint32_t doi1 = doi_case % h.ndoi, doi2 = doi_case / h.ndoi;
	const int2 zz = __ldg(h.zPairs + z_bin);
	d1 = a + static_cast<uint32_t>(zz.x) * h.dpr + doi1 * (h.dpr * h.rings);
	d2 = b + static_cast<uint32_t>(zz.y) * h.dpr + doi2 * (h.dpr * h.rings);
}

// Bin of the idx-th element of histogram subset `subset` (phi = subset mod
// numSubsets): BinIteratorRangeHistogram3D::getSafe (BinIterator.cpp:185-193).
__device__ __forceinline__ uint64_t h3SubsetBin(const H3Dev& h, uint64_t idx,
                                                uint64_t numPhiSubset,
                                                uint64_t numSubsets,
                                                uint64_t subset)
{
	const uint64_t per = numPhiSubset * h.numR;
	const uint64_t z_bin = idx / per;
	const uint64_t rem = idx % per;
	const uint64_t phi = (rem / h.numR) * numSubsets + subset;
	const uint64_t r = rem % h.numR;
	return z_bin * h.numPhi * h.numR + phi * h.numR + r;
}

uint64_t h3SubsetSize(const H3Host& h, uint64_t numSubsets, uint64_t subset,
                      uint64_t& numPhiSubset)
{
	numPhiSubset = h.numPhi / numSubsets;
	if (subset + numPhiSubset * numSubsets < h.numPhi)
		numPhiSubset += 1;
	return h.numR * numPhiSubset * h.numZBin;
}

// ------------------------------------------------------------ kernels ----
enum Kind
{
	K_SIDDON = 0,
	K_SIDDON_MR = 1,
	K_DD = 2,
	K_DD_PSF = 3
};

struct KParams
{
	Geom g;
	TofP tof;
	Psf psf;
	Scan scan;
	int numRays;
	// Multi-ray offsets of item indices 0 .. mrCount-1 (4 (numRays - 1)
	// uniforms each, as MultiRay::next draws them), or null.
	const float* mrTable;
	uint64_t mrCount;
};

// Endpoints (relative to the image centre) and orientations of event e.
__device__ __forceinline__ bool fetchEvent(const KParams& P, const Events& E,
                                           uint64_t e, float3& p1, float3& p2,
                                           float3& n1, float3& n2)
{
	if (E.d1 != nullptr)
	{
		const uint32_t a = __ldg(E.d1 + e), b = __ldg(E.d2 + e);
		// Invalid ids are counted by the caller and never dereferenced.
		if (a >= P.scan.numDets || b >= P.scan.numDets)
			return false;
		const float4 pa = __ldg(P.scan.pos + a), pb = __ldg(P.scan.pos + b);
		const float4 oa = __ldg(P.scan.ori + a), ob = __ldg(P.scan.ori + b);
		p1 = make_float3(pa.x, pa.y, pa.z);
		p2 = make_float3(pb.x, pb.y, pb.z);
		n1 = make_float3(oa.x, oa.y, oa.z);
		n2 = make_float3(ob.x, ob.y, ob.z);
	}
	else
	{
		const float* l = E.lor + e * 6;
		p1 = make_float3(__ldg(l + 0), __ldg(l + 1), __ldg(l + 2));
		p2 = make_float3(__ldg(l + 3), __ldg(l + 4), __ldg(l + 5));
		if (E.orient != nullptr)
		{
			const float* o = E.orient + e * 6;
			n1 = make_float3(__ldg(o + 0), __ldg(o + 1), __ldg(o + 2));
			n2 = make_float3(__ldg(o + 3), __ldg(o + 4), __ldg(o + 5));
		}
		else
		{
			n1 = make_float3(0.f, 0.f, 0.f);
			n2 = n1;
		}
	}
	if (E.mframe != nullptr)
	{
		const int mf = __ldg(E.mframe + e);
		if (mf >= 0 && static_cast<uint64_t>(mf) >= E.numMotion)
			return false;
		if (mf >= 0)
		{
			const float* m = E.motion + static_cast<int64_t>(mf) * 12;
			// transform_t layout: r00 r01 r02 tx r10 r11 r12 ty r20 r21 r22 tz.
			const float r00 = __ldg(m + 0), r01 = __ldg(m + 1), r02 = __ldg(m + 2);
			const float tx = __ldg(m + 3);
			const float r10 = __ldg(m + 4), r11 = __ldg(m + 5), r12 = __ldg(m + 6);
			const float ty = __ldg(m + 7);
			const float r20 = __ldg(m + 8), r21 = __ldg(m + 9), r22 = __ldg(m + 10);
			const float tz = __ldg(m + 11);
			// Matrix::operator*(Vector3D) then + translation (Matrix.cpp:177-186).
			float3 q1 = make_float3(r00 * p1.x + r01 * p1.y + r02 * p1.z,
			                        r10 * p1.x + r11 * p1.y + r12 * p1.z,
			                        r20 * p1.x + r21 * p1.y + r22 * p1.z);
			float3 q2 = make_float3(r00 * p2.x + r01 * p2.y + r02 * p2.z,
			                        r10 * p2.x + r11 * p2.y + r12 * p2.z,
			                        r20 * p2.x + r21 * p2.y + r22 * p2.z);
			p1 = make_float3(q1.x + tx, q1.y + ty, q1.z + tz);
			p2 = make_float3(q2.x + tx, q2.y + ty, q2.z + tz);
		}
	}
	const float3 off = make_float3(P.g.offx, P.g.offy, P.g.offz);
	p1 = f3sub(p1, off);
	p2 = f3sub(p2, off);
	return isfinite(p1.x) && isfinite(p1.y) && isfinite(p1.z) &&
	       isfinite(p2.x) && isfinite(p2.y) && isfinite(p2.z);
}

// Runs the configured projector over one event; endRay() after each ray.
// TILE: the image is in 4 x 2 tiles (tileOffset; single-ray Siddon only).
template <int KIND, bool TOF, bool COMP, bool TILE = false, typename Visit, typename EndRay>
__device__ __forceinline__ void projectEvent(const KParams& P, float3 p1,
                                             float3 p2, float3 n1, float3 n2,
                                             float tofv, uint64_t rid,
                                             bool forward, Visit& visit,
                                             EndRay& endRay, int part = 0,
                                             int parts = 1)
{
	static_assert(!TILE || KIND == K_SIDDON, "tiled images: single-ray Siddon");
	if constexpr (KIND == K_SIDDON)
	{
		siddonWalk<TOF, COMP, TILE>(P.g, p1, p2, P.tof, tofv, visit, 0.f, 1.f, part,
		                            parts);
		endRay();
	}
	else if constexpr (KIND == K_SIDDON_MR)
	{
		// The offsets come from the projector's table when it covers this
		// item index (same values), else from the generator.
		if (parts > 1)
		{
			// One lane per ray: this lane walks ray `part` only (none if part
			// >= numRays), its offsets read from the table, which the host
			// makes sure covers every item of the launch.  (parts is a
			// constant of the kernel, so the generator's code and state stay
			// out of these kernels.)
			if (part >= P.numRays)
				return;
			float3 a = p1, b = p2;
			if (part > 0)
			{
				MultiRay mr;
				mr.setDirs(n1, n2);
				const float4 t = __ldg(reinterpret_cast<const float4*>(P.mrTable) +
				                       rid * static_cast<uint64_t>(P.numRays - 1) + (part - 1));
				const float u[4] = {t.x, t.y, t.z, t.w};
				mr.offset(u, P.scan.crystalZ, P.scan.crystalTrans, a, b);
			}
			siddonWalk<TOF, COMP>(P.g, a, b, P.tof, tofv, visit);
			endRay();
			return;
		}
		MultiRay mr;
		const bool tab = P.mrTable != nullptr && rid < P.mrCount;
		if (tab)
			mr.setDirs(n1, n2);
		else
			mr.init(rid, n1, n2);
		const float* tu = tab ? P.mrTable + rid * 4 * static_cast<uint64_t>(P.numRays - 1)
		                      : nullptr;
		for (int k = 0; k < P.numRays; k++)
		{
			float3 a = p1, b = p2;
			if (k > 0)
			{
				float u[4];
				if (tab)
				{
					const float4 t = __ldg(reinterpret_cast<const float4*>(tu) + (k - 1));
					u[0] = t.x;
					u[1] = t.y;
					u[2] = t.z;
					u[3] = t.w;
				}
				else
				{
					mr.next(u);
				}
				mr.offset(u, P.scan.crystalZ, P.scan.crystalTrans, a, b);
			}
			siddonWalk<TOF, COMP>(P.g, a, b, P.tof, tofv, visit);
			endRay();
		}
	}
	else
	{
		ddWalk<TOF, KIND == K_DD_PSF, COMP && KIND == K_DD_PSF, COMP>(P.g, p1, p2, n1, n2, P.scan.crystalTrans,
		                              P.scan.crystalZ, P.tof, tofv, P.psf,
		                              forward, visit, part, parts);
		endRay();
	}
}

// Forward sum of one event (or of piece `part` of `parts` of a single-ray
// Siddon walk): per-ray partial sums added ray by ray; mirror mode sums in
// traversal order, compensated mode uses Kahan summation.  With TRACK, maxw
// receives the largest |weight| of the event's rays (the sum itself is
// computed exactly as without TRACK).
// VEC: the image is read as aligned float4 groups, and consecutive
// crossings inside one group (x steps) reuse the group held in registers.
template <int KIND, bool TOF, bool COMP, bool TRACK = false, bool VEC = false,
          bool TILE = false>
__device__ __forceinline__ float forwardEvent(const KParams& P,
                                              const float* __restrict__ img,
                                              float3 p1, float3 p2, float3 n1,
                                              float3 n2, float tofv,
                                              uint64_t rid,
                                              float* maxw = nullptr,
                                              int part = 0, int parts = 1)
{
	float acc = 0.f, ray = 0.f, comp = 0.f, mw = 0.f;
	int gb = -1;
	float4 q4 = make_float4(0.f, 0.f, 0.f, 0.f);
	auto fetch = [&](int o) -> float
	{
		if constexpr (VEC)
		{
			const int g = o & ~3;
			if (g != gb)
			{
				q4 = __ldg(reinterpret_cast<const float4*>(img + g));
				gb = g;
			}
			const int l = o & 3;
			return l == 0 ? q4.x : (l == 1 ? q4.y : (l == 2 ? q4.z : q4.w));
		}
		else
		{
			return __ldg(img + o);
		}
	};
	auto visit = [&](int o, float w)
	{
		if constexpr (TRACK)
			mw = fmaxf(mw, fabsf(w));
		if constexpr (COMP)
		{
			const float y = __fmaf_rn(w, fetch(o), -comp);
			const float t = ray + y;
			comp = (t - ray) - y;
			ray = t;
		}
		else
		{
			ray += w * fetch(o);
		}
	};
	auto endRay = [&]
	{
		acc += ray;
		ray = 0.f;
		comp = 0.f;
	};
	projectEvent<KIND, TOF, COMP, TILE>(P, p1, p2, n1, n2, tofv, rid, true, visit,
	                                    endRay, part, parts);
	// One lane per ray (parts > 1): the caller adds the rays' sums in ray
	// order and divides (rayGroupMean).
	if constexpr (KIND == K_SIDDON_MR)
		if (parts == 1)
			acc = acc / static_cast<float>(P.numRays);
	if constexpr (TRACK)
		*maxw = mw;
	return acc;
}

// Largest |weight| along the event's rays (a walk without image reads).
template <int KIND, bool TOF, bool COMP>
__device__ __forceinline__ float maxWeightEvent(const KParams& P, float3 p1,
                                                float3 p2, float3 n1, float3 n2,
                                                float tofv, uint64_t rid)
{
	float mw = 0.f;
	auto visit = [&](int, float w) { mw = fmaxf(mw, fabsf(w)); };
	auto endRay = [] {};
	projectEvent<KIND, TOF, COMP>(P, p1, p2, n1, n2, tofv, rid, false, visit,
	                              endRay);
	return mw;
}

// ------------------------------------------- deterministic back projection --
// Two passes.  Pass 1 reduces M = max over events of |v_e| * max_k |w_ek|
// (v_e the value back-projected along event e, w_ek its voxel weights; for
// multi-ray, the rays of one event add at most |v_e| max|w| to a voxel).  Any
// voxel then receives at most n * M in magnitude from the n events of the
// call.  Pass 2 scatters round(v_e * w_ek * 2^s) into 64-bit integers with
// 2^s the largest power of two for which n * M * 2^s <= 2^61, so the integer
// sums cannot overflow (the roundings add at most numRays * n / 2 < 2^62).
// Integer addition is associative: the image is the same whatever order the
// atomics land in, and equal to the exact sum to within n/2 units of 2^-s.
struct Fixed
{
	unsigned long long* acc;  // nvox * nt fixed-point image (zeroed by the caller)
	const unsigned* maxBits;  // M as float bits (pass 1 result)
	uint64_t n;               // events (bins) of the call
};

// Exponent k with n * M < 2^k; 0x7fffffff when M is zero or not finite.
__device__ __forceinline__ int fixedExponent(unsigned maxBits, uint64_t n)
{
	const double b = static_cast<double>(n) * static_cast<double>(__uint_as_float(maxBits));
	if (!(b > 0.0) || !isfinite(b))
		return 0x7fffffff;
	int k;
	frexp(b, &k);
	return k;
}

// 2^(61 - k): exact scale of the fixed-point contributions (0 if none).
__device__ __forceinline__ double fixedScale(const Fixed& F)
{
	const int k = fixedExponent(*F.maxBits, F.n);
	return k == 0x7fffffff ? 0.0 : ldexp(1.0, 61 - k);
}

// Warp max of a non-negative float (as bits) folded into *out by lane 0.  All
// 32 lanes of the warp must call it.
__device__ __forceinline__ void warpMaxInto(unsigned* out, float b)
{
	const unsigned bits = __reduce_max_sync(0xffffffffu, __float_as_uint(b));
	if ((threadIdx.x & 31) == 0 && bits != 0u)
		atomicMax(out, bits);
}

// VEC: contributions to one aligned group of 4 voxels (consecutive x steps)
// are summed in registers and sent as one red.global.add.v4.f32 (the other
// lanes add zero), which cuts the L2 reduction requests.
__device__ __forceinline__ void redV4(float* p, float4 v)
{
	asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};"
	             :: "l"(p), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w) : "memory");
}

// The same for an aligned pair of voxels (8-byte aligned p).
__device__ __forceinline__ void redV2(float* p, float2 v)
{
	asm volatile("red.global.add.v2.f32 [%0], {%1, %2};"
	             :: "l"(p), "f"(v.x), "f"(v.y) : "memory");
}

// VEC 1: the group is summed in registers; VEC 2: the group's four values
// are staged in this thread's shared-memory slots (vslot[l * vstride]; a
// single-ray walk visits each voxel once, so a slot is written at most once
// per group) and read back only to send the group; VEC 3: pairs of voxels
// instead of groups of four, held in registers and sent as one
// red.global.add.v2.f32 (more requests than VEC 1, fewer instructions per
// visit).
template <int KIND, bool TOF, bool COMP, bool FIX = false, int VEC = 0,
          bool TILE = false>
__device__ __forceinline__ void backwardEvent(const KParams& P,
                                              float* __restrict__ img,
                                              float v, float3 p1, float3 p2,
                                              float3 n1, float3 n2, float tofv,
                                              uint64_t rid,
                                              unsigned long long* fix = nullptr,
                                              double scale = 0.0, int part = 0,
                                              int parts = 1,
                                              float* vslot = nullptr,
                                              int vstride = 0)
{
	if constexpr (KIND == K_SIDDON_MR)
		v = v / static_cast<float>(P.numRays);
	auto endRay = [] {};
	if constexpr (FIX)
	{
		const double vs = static_cast<double>(v) * scale;
		auto visit = [&](int o, float w)
		{
			const long long q = __double2ll_rn(vs * static_cast<double>(w));
			atomicAdd(fix + o, static_cast<unsigned long long>(q));
		};
		projectEvent<KIND, TOF, COMP>(P, p1, p2, n1, n2, tofv, rid, false, visit,
		                              endRay, part, parts);
	}
	else if constexpr (VEC == 2)
	{
		// Multi-ray: flush ends every ray, so a group never spans two rays.
		static_assert(KIND == K_SIDDON || KIND == K_SIDDON_MR,
		              "slots hold one value per voxel of one ray");
		int gb = -1;
		auto send = [&]
		{
			const float4 a = make_float4(vslot[0], vslot[vstride], vslot[2 * vstride],
			                             vslot[3 * vstride]);
			redV4(img + gb, a);
		};
		auto visit = [&](int o, float w)
		{
			const int g = o & ~3;
			if (g != gb)
			{
				if (gb >= 0)
					send();
				vslot[0] = 0.f;
				vslot[vstride] = 0.f;
				vslot[2 * vstride] = 0.f;
				vslot[3 * vstride] = 0.f;
				gb = g;
			}
			vslot[(o & 3) * vstride] = v * w;
		};
		auto flush = [&]
		{
			if (gb >= 0)
				send();
			gb = -1;
		};
		projectEvent<KIND, TOF, COMP, TILE>(P, p1, p2, n1, n2, tofv, rid, false, visit,
		                                    flush, part, parts);
	}
	else if constexpr (VEC == 1)
	{
		static_assert(KIND == K_SIDDON || KIND == K_SIDDON_MR,
		              "lanes hold one value per voxel of one ray");
		int gb = -1;
		float4 a4 = make_float4(0.f, 0.f, 0.f, 0.f);
		auto visit = [&](int o, float w)
		{
			const float c = v * w;
			const int g = o & ~3;
			const bool nw = g != gb;
			if (nw && gb >= 0)
				redV4(img + gb, a4);
			gb = g;
			// A single-ray walk visits each voxel once: a lane is set, never
			// summed, inside a group (and cleared when a new group starts).
			const int l = o & 3;
			a4.x = l == 0 ? c : (nw ? 0.f : a4.x);
			a4.y = l == 1 ? c : (nw ? 0.f : a4.y);
			a4.z = l == 2 ? c : (nw ? 0.f : a4.z);
			a4.w = l == 3 ? c : (nw ? 0.f : a4.w);
		};
		auto flush = [&]
		{
			if (gb >= 0)
				redV4(img + gb, a4);
			gb = -1;
		};
		projectEvent<KIND, TOF, COMP, TILE>(P, p1, p2, n1, n2, tofv, rid, false, visit,
		                                    flush, part, parts);
	}
	else if constexpr (VEC == 3)
	{
		static_assert(KIND == K_SIDDON || KIND == K_SIDDON_MR,
		              "lanes hold one value per voxel of one ray");
		int gb = -1;
		float2 a2 = make_float2(0.f, 0.f);
		auto visit = [&](int o, float w)
		{
			const float c = v * w;
			const int g = o & ~1;
			const bool nw = g != gb;
			if (nw && gb >= 0)
				redV2(img + gb, a2);
			gb = g;
			// Set, never summed, inside a pair (cleared when a new one starts).
			const bool hi = (o & 1) != 0;
			a2.x = hi ? (nw ? 0.f : a2.x) : c;
			a2.y = hi ? c : (nw ? 0.f : a2.y);
		};
		auto flush = [&]
		{
			if (gb >= 0)
				redV2(img + gb, a2);
			gb = -1;
		};
		projectEvent<KIND, TOF, COMP, TILE>(P, p1, p2, n1, n2, tofv, rid, false, visit,
		                                    flush, part, parts);
	}
	else
	{
		auto visit = [&](int o, float w) { atomicAdd(img + o, v * w); };
		projectEvent<KIND, TOF, COMP, TILE>(P, p1, p2, n1, n2, tofv, rid, false, visit,
		                                    endRay, part, parts);
	}
}

enum Op
{
	OP_FWD = 0,
	OP_BWD = 1,
	OP_EM = 2,
	OP_COUNT = 3
};

// Sum over the TPL lanes that share one event (all of them active).
template <int TPL>
__device__ __forceinline__ float groupSum(float v)
{
	if constexpr (TPL > 1)
	{
		const unsigned lane = threadIdx.x & 31u;
		const unsigned mask = ((1u << TPL) - 1u) << (lane & ~static_cast<unsigned>(TPL - 1));
		// xor butterfly: every lane adds the same pairs, so all TPL lanes end
		// with the same bits.
		for (int o = TPL / 2; o > 0; o >>= 1)
			v += __shfl_xor_sync(mask, v, o);
	}
	return v;
}

// Multi-ray event held by TPL lanes, lane r with the sum of ray r: the rays'
// sums added in ray order from 0 and divided by the number of rays, as one
// thread walking the rays one after the other computes them (same bits, in
// every lane of the group).
template <int TPL>
__device__ __forceinline__ float rayGroupMean(float ray, int numRays)
{
	const unsigned lane = threadIdx.x & 31u;
	const unsigned base = lane & ~static_cast<unsigned>(TPL - 1);
	const unsigned mask = (TPL == 32 ? 0xffffffffu : ((1u << TPL) - 1u)) << base;
	float acc = 0.f;
#pragma unroll
	for (int r = 0; r < TPL; r++)
	{
		const float x = __shfl_sync(mask, ray, base + r);
		if (r < numRays)
			acc += x;
	}
	return acc / static_cast<float>(numRays);
}

// One event per TPL threads.  TPL > 1, single-ray Siddon (compensated
// arithmetic): lane j of the group walks piece j of the ray and the forward
// sum is reduced over the group.  TPL > 1, multi-ray Siddon: lane r walks
// ray r, the forward sums are added in ray order (rayGroupMean), the same
// bits as one thread walking the rays in turn.  Compensated Siddon, and
// multi-ray with one lane per ray: 1024 threads per SM (64 registers per
// thread, 32 warps) whatever the block size; mirror Siddon and multi-ray with
// one thread per event: 768 (80 registers: the mirror walk keeps three voxel
// coordinates and a row offset; C2 TOF EM pass 2.95 -> 2.80 ms per 5M events,
// while the compensated walk is faster at 1024, 2.05 vs 2.13 ms); the other
// projectors keep the compiler's register choice.  FIX (OP_BWD, OP_EM):
// pass 2 of the deterministic back projection.  TILE: the images are in
// 4 x 2 tiles (tileOffset).
template <int OP, int KIND, bool TOF, bool COMP, bool FIX = false,
          int BLOCK = kBlock, int TPL = 1, int VEC = 0, bool TILE = false>
__global__ void __launch_bounds__(BLOCK, ((KIND == K_SIDDON && COMP) ||
                                          (KIND == K_SIDDON_MR && TPL > 1))
                                             ? 1024 / BLOCK
                                             : ((KIND == K_SIDDON || KIND == K_SIDDON_MR)
                                                    ? 768 / BLOCK
                                                    : 1))
    k_events(KParams P, Events E, Range R, const float* __restrict__ in,
             float* __restrict__ out, float globalScale, float denomThr,
             unsigned long long* err, Fixed F)
{
	static_assert(TPL == 1 || (KIND == K_SIDDON && COMP && !FIX && OP != OP_COUNT) ||
	                  (KIND == K_SIDDON_MR && !FIX && OP != OP_COUNT),
	              "several threads per LOR: single-ray Siddon (compensated) or one "
	              "lane per ray of a multi-ray Siddon");
	static_assert(!TILE || (KIND == K_SIDDON && TPL == 1 && !FIX && OP != OP_COUNT),
	              "tiled images: single-ray Siddon, one thread per LOR, float scatter");
	// Forward sum of the event from the TPL lanes' partial sums.
	auto eventSum = [&](float v) -> float
	{
		if constexpr (KIND == K_SIDDON_MR && TPL > 1)
			return rayGroupMean<TPL>(v, P.numRays);
		else
			return groupSum<TPL>(v);
	};
	// One item per thread group: a warp's threads stay converged across items
	// (a grid-stride loop lets them drift apart between items).
	const uint64_t gt = static_cast<uint64_t>(blockIdx.x) * BLOCK + threadIdx.x;
	const uint64_t k = gt / TPL;
	const int part = static_cast<int>(gt % TPL);
	// Shared-memory slots of the staged float4 reductions (VEC bit 2); VEC
	// bit 3: float2 pair reductions.
	constexpr int kRedMode = (VEC & 4) ? 2 : ((VEC & 2) ? 1 : ((VEC & 8) ? 3 : 0));
	float* vslot = nullptr;
	if constexpr (kRedMode == 2)
	{
		__shared__ float vacc[4 * BLOCK];
		vslot = vacc + threadIdx.x;
	}
	if (k < R.count)
	{
		const uint64_t e = R.start + k * R.stride;
		const int frame = E.frame ? __ldg(E.frame + e) : 0;
		float3 p1, p2, n1, n2;
		if (frame < 0 || frame >= P.g.nt || !fetchEvent(P, E, e, p1, p2, n1, n2))
		{
			if (part == 0)
			{
				if (frame >= 0)
					atomicAdd(err, 1ULL);
				if constexpr (OP == OP_FWD)
					out[e] = 0.f;
				if constexpr (OP == OP_EM)
					if (E.model)
						E.model[e] = 0.f;
				if constexpr (OP == OP_COUNT)
					reinterpret_cast<uint32_t*>(out)[e] = 0u;
			}
			return;
		}
		const float tofv = TOF ? __ldg(E.tof + e) : 0.f;
		const int64_t fo = static_cast<int64_t>(frame) * P.g.nvox;
		if constexpr (OP == OP_COUNT)
		{
			unsigned c = 0;
			auto visit = [&](int, float) { c++; };
			auto endRay = [] {};
			projectEvent<KIND, TOF, COMP>(P, p1, p2, n1, n2, tofv, k, true, visit,
			                              endRay);
			reinterpret_cast<uint32_t*>(out)[e] = c;
		}
		else if constexpr (OP == OP_FWD)
		{
			const float v = eventSum(forwardEvent<KIND, TOF, COMP, false, (VEC & 1) != 0, TILE>(
			    P, in + fo, p1, p2, n1, n2, tofv, k, nullptr, part, TPL));
			if (part == 0)
				out[e] = v;
		}
		else if constexpr (OP == OP_BWD)
		{
			if constexpr (FIX)
				backwardEvent<KIND, TOF, COMP, true>(P, nullptr, __ldg(in + e), p1,
				                                     p2, n1, n2, tofv, k,
				                                     F.acc + fo, fixedScale(F));
			else
				backwardEvent<KIND, TOF, COMP, false, kRedMode, TILE>(
				    P, out + fo, __ldg(in + e), p1, p2, n1, n2, tofv, k, nullptr, 0.0,
				    part, TPL, vslot, BLOCK);
		}
		else
		{
			const float m = E.meas ? __ldg(E.meas + e) : 1.0f;
			const float s = E.sens ? __ldg(E.sens + e) : 1.0f;
			const float a = E.att ? __ldg(E.att + e) : 1.0f;
			if (m == 0.f || s == 0.f || a == 0.f)
			{
				if (E.model && part == 0)
					E.model[e] = 0.f;
				return;
			}
			float u = eventSum(forwardEvent<KIND, TOF, COMP, false, (VEC & 1) != 0, TILE>(
			    P, in + fo, p1, p2, n1, n2, tofv, k, nullptr, part, TPL));
			u *= s;
			u *= a;
			u *= globalScale;
			if (E.add)
				u += __ldg(E.add + e);
			if (E.model && part == 0)
				E.model[e] = u;
			if (fabsf(u) > denomThr)
			{
				u = m / u;
				u *= s;
				u *= a;
				u *= globalScale;
				if constexpr (FIX)
					backwardEvent<KIND, TOF, COMP, true>(P, nullptr, u, p1, p2, n1,
					                                     n2, tofv, k, F.acc + fo,
					                                     fixedScale(F));
				else
					backwardEvent<KIND, TOF, COMP, false, kRedMode, TILE>(P, out + fo, u, p1, p2,
					                                                n1, n2, tofv, k, nullptr,
					                                                0.0, part, TPL, vslot,
					                                                BLOCK);
			}
		}
	}
}

// Diagnostics: the (offset, weight) visits of each event's walk in walk
// order, item k of the range at offs/wts[k * cap ...] (at most cap of them),
// the number of visits in counts[k]; offsets within the event's frame.
template <int KIND, bool TOF, bool COMP>
__global__ void __launch_bounds__(kBlock)
    k_trace(KParams P, Events E, Range R, uint32_t cap, int32_t* __restrict__ offs,
            float* __restrict__ wts, uint32_t* __restrict__ counts,
            unsigned long long* err)
{
	const uint64_t k = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	if (k >= R.count)
		return;
	const uint64_t e = R.start + k * R.stride;
	const int frame = E.frame ? __ldg(E.frame + e) : 0;
	float3 p1, p2, n1, n2;
	if (frame < 0 || frame >= P.g.nt || !fetchEvent(P, E, e, p1, p2, n1, n2))
	{
		if (frame >= 0)
			atomicAdd(err, 1ULL);
		counts[k] = 0u;
		return;
	}
	const float tofv = TOF ? __ldg(E.tof + e) : 0.f;
	int32_t* o = offs + k * cap;
	float* w = wts + k * cap;
	uint32_t c = 0;
	auto visit = [&](int off, float wt)
	{
		if (c < cap)
		{
			o[c] = off;
			w[c] = wt;
		}
		c++;
	};
	auto endRay = [] {};
	projectEvent<KIND, TOF, COMP>(P, p1, p2, n1, n2, tofv, k, true, visit, endRay);
	counts[k] = c;
}

// Pass 1 of the deterministic back projection of k_events<OP_BWD / OP_EM>:
// folds |v_e| * max|w| of every event that pass 2 back-projects into
// *maxBits.  The EM value v_e is computed exactly as in k_events (same
// forward sum, same correction order).  Invalid events are left to pass 2,
// which counts them.
template <bool EM, int KIND, bool TOF, bool COMP>
__global__ void __launch_bounds__(kBlock, KIND == K_SIDDON ? 4 : 1)
    k_events_bound(KParams P, Events E, Range R, const float* __restrict__ in,
                   float globalScale, float denomThr, unsigned* maxBits)
{
	const uint64_t k = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	float b = 0.f;
	if (k < R.count)
	{
		const uint64_t e = R.start + k * R.stride;
		const int frame = E.frame ? __ldg(E.frame + e) : 0;
		float3 p1, p2, n1, n2;
		if (frame >= 0 && frame < P.g.nt && fetchEvent(P, E, e, p1, p2, n1, n2))
		{
			const float tofv = TOF ? __ldg(E.tof + e) : 0.f;
			if constexpr (!EM)
			{
				const float v = __ldg(in + e);
				if (v != 0.f)
					b = fabsf(v) * maxWeightEvent<KIND, TOF, COMP>(P, p1, p2, n1, n2,
					                                                tofv, k);
			}
			else
			{
				const int64_t fo = static_cast<int64_t>(frame) * P.g.nvox;
				const float m = E.meas ? __ldg(E.meas + e) : 1.0f;
				const float s = E.sens ? __ldg(E.sens + e) : 1.0f;
				const float a = E.att ? __ldg(E.att + e) : 1.0f;
				if (m != 0.f && s != 0.f && a != 0.f)
				{
					float mw = 0.f;
					float u = forwardEvent<KIND, TOF, COMP, true>(
					    P, in + fo, p1, p2, n1, n2, tofv, k, &mw);
					u *= s;
					u *= a;
					u *= globalScale;
					if (E.add)
						u += __ldg(E.add + e);
					if (fabsf(u) > denomThr)
					{
						u = m / u;
						u *= s;
						u *= a;
						u *= globalScale;
						b = fabsf(u) * mw;
					}
				}
			}
		}
	}
	// NaN bits order above every finite value, so a NaN bound is kept.
	warpMaxInto(maxBits, b != b ? __uint_as_float(0x7fffffffu) : b);
}

// out[i] += fixed-point image / 2^s (NaN everywhere if the bound was not
// finite: a value back-projected was NaN or infinite).
__global__ void k_fixed_finish(const unsigned long long* __restrict__ acc,
                               uint64_t n, Fixed F, float* __restrict__ out)
{
	const int k = fixedExponent(*F.maxBits, F.n);
	const bool bad = k == 0x7fffffff && *F.maxBits != 0u;
	if (k == 0x7fffffff && !bad)
		return;  // nothing was back-projected
	const double inv = bad ? 0.0 : ldexp(1.0, k - 61);
	const uint64_t nthreads = static_cast<uint64_t>(gridDim.x) * blockDim.x;
	for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	     i < n; i += nthreads)
	{
		if (bad)
			out[i] = __int_as_float(0x7fffffff);
		else
			out[i] += static_cast<float>(
			    static_cast<double>(static_cast<long long>(acc[i])) * inv);
	}
}

// Estimated crossings per event (crossingEstimate) for the event ordering.
template <bool TOF>
__global__ void k_count_estimate(KParams P, Events E, uint64_t n,
                                 uint32_t* __restrict__ out)
{
	const uint64_t nthreads = static_cast<uint64_t>(gridDim.x) * blockDim.x;
	for (uint64_t e = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	     e < n; e += nthreads)
	{
		const int frame = E.frame ? __ldg(E.frame + e) : 0;
		float3 p1, p2, n1, n2;
		uint32_t c = 0;
		if (frame >= 0 && frame < P.g.nt && fetchEvent(P, E, e, p1, p2, n1, n2))
			c = crossingEstimate<TOF>(P.g, p1, p2, P.tof, TOF ? __ldg(E.tof + e) : 0.f);
		out[e] = c;
	}
}

__global__ void k_box_init(int* box)
{
	if (threadIdx.x < 6)
		box[threadIdx.x] = threadIdx.x < 3 ? INT_MAX : -1;
}

// Bounding box (voxel indices, inclusive) of the non-zero voxels of an image:
// box = {min x, min y, min z, max x, max y, max z}; initialised to an empty
// box by the caller.
__global__ void k_support_box(const float* __restrict__ img, Geom g, int* box)
{
	const uint64_t nthreads = static_cast<uint64_t>(gridDim.x) * blockDim.x;
	int mn[3] = {INT_MAX, INT_MAX, INT_MAX}, mx[3] = {-1, -1, -1};
	for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	     i < static_cast<uint64_t>(g.nvox); i += nthreads)
	{
		if (__ldg(img + i) != 0.f)
		{
			const int x = static_cast<int>(i % g.nx);
			const int y = static_cast<int>((i / g.nx) % g.ny);
			const int z = static_cast<int>(i / g.nxy);
			mn[0] = min(mn[0], x); mn[1] = min(mn[1], y); mn[2] = min(mn[2], z);
			mx[0] = max(mx[0], x); mx[1] = max(mx[1], y); mx[2] = max(mx[2], z);
		}
	}
	for (int k = 0; k < 3; k++)
	{
		for (int o = 16; o > 0; o >>= 1)
		{
			mn[k] = min(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
			mx[k] = max(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
		}
	}
	if ((threadIdx.x & 31) == 0 && mx[0] >= 0)
	{
		for (int k = 0; k < 3; k++)
		{
			atomicMin(box + k, mn[k]);
			atomicMax(box + 3 + k, mx[k]);
		}
	}
}

// Moves the endpoints of fetchEvent (relative to the reconstruction grid) to
// the attenuation grid and gives the ray's parametric window inside the
// mu-map's non-zero bounding box: only voxels there contribute, so the walk
// is limited to it.
__device__ __forceinline__ void attShift(const KParams& P, const Geom& mu,
                                         float3& p1, float3& p2)
{
	const float3 fix = make_float3(P.g.offx - mu.offx, P.g.offy - mu.offy,
	                               P.g.offz - mu.offz);
	p1 = make_float3(p1.x + fix.x, p1.y + fix.y, p1.z + fix.z);
	p2 = make_float3(p2.x + fix.x, p2.y + fix.y, p2.z + fix.z);
}

__device__ __forceinline__ void attWindow(const KParams& P, const Geom& mu,
                                          const int* box, float3& p1, float3& p2,
                                          float& wlo, float& whi)
{
	attShift(P, mu, p1, p2);
	boxWindow(mu, box, p1, p2, wlo, whi);
}

// Walk-length bucket of each item of the range for the attenuation walks:
// an O(1) estimate of the voxel planes the ray crosses inside its window in
// the mu-map's support box, in buckets of 4 (255 = 1020 or more), with the
// item's index for the sort.  The events arrive in reconstruction order
// (subset, TOF-window length, LOR), which says nothing about the length of
// their full chords through the mu-map; a warp of such walks ran about 10 of
// its 32 lanes.
__global__ void k_att_keys(KParams P, Geom mu, Events E, Range R,
                           const int* __restrict__ box, uint8_t* __restrict__ keys,
                           uint32_t* __restrict__ idx)
{
	const uint64_t nthreads = static_cast<uint64_t>(gridDim.x) * blockDim.x;
	for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	     i < R.count; i += nthreads)
	{
		const uint64_t e = R.start + i * R.stride;
		float3 p1, p2, n1, n2;
		unsigned c = 0;
		if (fetchEvent(P, E, e, p1, p2, n1, n2))
		{
			float wlo, whi;
			attWindow(P, mu, box, p1, p2, wlo, whi);
			if (wlo < whi)
			{
				auto planes = [&](float p, float d, float q0, float dq) -> unsigned
				{
					if (d == 0.f)
						return 0u;
					const float u = floorf((p + wlo * d - q0) / dq);
					const float v = floorf((p + whi * d - q0) / dq);
					return static_cast<unsigned>(fminf(fabsf(v - u), 65536.f));
				};
				c = 1u + planes(p1.x, p2.x - p1.x, -0.5f * mu.lx, mu.vx) +
				    planes(p1.y, p2.y - p1.y, -0.5f * mu.ly, mu.vy) +
				    planes(p1.z, p2.z - p1.z, -0.5f * mu.lz, mu.vz);
			}
		}
		keys[i] = static_cast<uint8_t>(min(c >> 2, 255u));
		idx[i] = static_cast<uint32_t>(i);
	}
}

// Attenuation factor per event: exp(-0.1 * line integral of mu), walked with
// the projector's arithmetic (COMP: compensated walk).
// Crossings per batch of mu reads: 4 for the compensated walk, 8 for the
// mirror walk (5M C2 walks: 1.21 ms at 4 vs 1.22 at 8 and 1.30 at 2
// compensated; 3.50 ms at 8 vs 3.65 at 4 mirror).
template <bool COMP>
__host__ __device__ constexpr int attBatch()
{
	return COMP ? 4 : 8;
}
constexpr int kAttBlocksPerSM = 4;
template <bool COMP>
__global__ void __launch_bounds__(kBlock, kAttBlocksPerSM)
    k_attenuation(KParams P, Geom mu, Events E, Range R,
                  const float* __restrict__ muImg, const int* __restrict__ box,
                  float* __restrict__ out, unsigned long long* err,
                  const uint32_t* __restrict__ order)
{
	// One item per thread: a warp's threads stay converged across items
	// (a grid-stride loop lets them drift apart between items).  With order,
	// thread i walks item order[i] (items grouped by walk length, see
	// k_att_keys), so that the lanes of a warp walk similar lengths, and the
	// warp walks its rays in lock step (siddonWalkWarp): every lane of the
	// warp reaches the walk, lanes without a ray as idle participants.
	const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	uint64_t e = 0;
	float3 p1 = make_float3(0.f, 0.f, 0.f), p2 = p1, n1, n2;
	bool ok = false;
	if (i < R.count)
	{
		const uint64_t k = order ? __ldg(order + i) : i;
		e = R.start + k * R.stride;
		ok = fetchEvent(P, E, e, p1, p2, n1, n2);
		if (!ok)
		{
			atomicAdd(err, 1ULL);
			out[e] = 0.f;
		}
	}
	float wlo = 0.f, whi = 1.f;
	if (ok)
	{
		if constexpr (COMP)
		{
			attWindow(P, mu, box, p1, p2, wlo, whi);
		}
		else
		{
			// Mirror arithmetic walks the whole chord, as the reference's
			// Siddon projection of the mu-map does
			// (Corrector::getAttenuationFactorFromAttenuationImage,
			// src/recon/Corrector.cpp:601-611): a walk that starts at the
			// support box places its first voxel from a different first
			// segment, which in FP32 can round onto the other side of a plane.
			attShift(P, mu, p1, p2);
		}
	}
	// Batches of attBatch crossings: their mu reads are all in flight before
	// the first is added (the walk itself needs none of them), and the sum
	// still runs in walk order.
	float acc = 0.f;
	constexpr int kAttBatch = attBatch<COMP>();
	auto consume = [&](const int (&o)[kAttBatch], const float (&w)[kAttBatch])
	{
		float m[kAttBatch];
#pragma unroll
		for (int k = 0; k < kAttBatch; k++)
			m[k] = o[k] >= 0 ? __ldg(muImg + o[k]) : 0.f;
#pragma unroll
		for (int k = 0; k < kAttBatch; k++)
			if (o[k] >= 0)
				acc += w[k] * m[k];
	};
	siddonWalkWarpBatched<false, COMP, kAttBatch>(ok && wlo < whi, mu, p1, p2, P.tof,
	                                              0.f, consume, wlo, whi);
	if (ok)
		out[e] = expf(-acc * 0.1f);
}

__global__ void __launch_bounds__(kBlock)
    k_gather_histo(KParams P, H3Dev H, Events E, Range R,
                   const float* __restrict__ histo, int invert,
                   float* __restrict__ out, unsigned long long* err)
{
	// One item per thread: a warp's threads stay converged across items
	// (a grid-stride loop lets them drift apart between items).
	const uint64_t k = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	if (k < R.count)
	{
		const uint64_t e = R.start + k * R.stride;
		uint64_t b;
		float v = 0.f;
		if (h3Bin(H, __ldg(E.d1 + e), __ldg(E.d2 + e), b))
		{
			v = __ldg(histo + b);
			if (invert && v != 0.f)
				v = 1.0f / v;
		}
		else
		{
			atomicAdd(err, 1ULL);
		}
		out[e] = v;
	}
}

// Per-event product of crystal factors eff[d1] * eff[d2]: the LOR
// sensitivity of a normalisation made of per-crystal efficiencies (the value a
// Histogram3D filled with eff[d1] * eff[d2] holds for the event's bin).
// Detector ids outside the scanner give 0 and are counted.
__global__ void __launch_bounds__(kBlock)
    k_gather_crystal(uint32_t numDets, Events E, Range R,
                     const float* __restrict__ eff, float* __restrict__ out,
                     unsigned long long* err)
{
	const uint64_t k = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	if (k < R.count)
	{
		const uint64_t e = R.start + k * R.stride;
		const uint32_t a = __ldg(E.d1 + e), b = __ldg(E.d2 + e);
		float v = 0.f;
		if (a < numDets && b < numDets)
			v = __ldg(eff + a) * __ldg(eff + b);
		else
			atomicAdd(err, 1ULL);
		out[e] = v;
	}
}

// Histogram-bin kernels: sensitivity back projection and histogram EM.
// MODE H_BOUND is pass 1 and H_FIX pass 2 of the deterministic back
// projection (see Fixed); H_PLAIN scatters floats.
enum HistoMode
{
	H_PLAIN = 0,
	H_BOUND = 1,
	H_FIX = 2
};

// Blocks per SM of the compensated DD + PSF histogram EM kernel (several
// threads per bin).
constexpr int kDDPsfBlocksPerSM = 2;
template <int KIND, bool EM, int MODE = H_PLAIN, bool COMP = false, int TPL = 1>
__global__ void __launch_bounds__(kBlock, (KIND == K_DD_PSF && TPL > 1) ? kDDPsfBlocksPerSM : 1)
    k_histo(KParams P, H3Dev H, uint64_t count, uint64_t numPhiSubset,
            uint64_t numSubsets, uint64_t subset, const float* __restrict__ img,
            float* __restrict__ out, const float* __restrict__ meas,
            const float* __restrict__ sensH, const float* __restrict__ acfH,
            const float* __restrict__ addH, Geom mu,
            const float* __restrict__ muImg, float globalScale, float denomThr,
            Fixed F, unsigned* maxBits, const uint64_t* __restrict__ list,
            const float* __restrict__ crystalEff)
{
	static_assert(TPL == 1 || (KIND == K_DD_PSF && EM && MODE == H_PLAIN && COMP),
	              "several threads per bin: compensated DD + PSF histogram EM");
	// One item per TPL threads: a warp's threads stay converged across items
	// (a grid-stride loop lets them drift apart between items).  With a list,
	// item t is the subset-local bin index list[t] (count = list length), so
	// that warps hold only the bins that do work.  TPL > 1: lane j of a group
	// walks piece j of the bin's rows; the forward partial sums are added over
	// the group, which then shares the EM ratio.
	const uint64_t gt = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	const uint64_t t = gt / TPL;
	const int part = static_cast<int>(gt % TPL);
	float bound = 0.f;  // H_BOUND: |v| * max|w| of this bin
	do
	{
		if (t >= count)
			break;
		const uint64_t k = list ? __ldg(list + t) : t;
		const uint64_t bin = h3SubsetBin(H, k, numPhiSubset, numSubsets, subset);
		uint32_t d1, d2;
		h3Pair(H, bin, d1, d2);
		if (d1 == 0 && d2 == 0)
			break;
		const float m = EM ? __ldg(meas + bin) : 1.0f;
		if (EM && m == 0.f)
			break;
		// LOR sensitivity: a histogram value, or the product of the two
		// crystals' factors (the same FP32 product a histogram of them holds).
		const float s = sensH ? __ldg(sensH + bin) :
		                (crystalEff ? __ldg(crystalEff + d1) * __ldg(crystalEff + d2) : 1.0f);
		const float4 pa = __ldg(P.scan.pos + d1), pb = __ldg(P.scan.pos + d2);
		const float4 oa = __ldg(P.scan.ori + d1), ob = __ldg(P.scan.ori + d2);
		float3 p1 = make_float3(pa.x, pa.y, pa.z), p2 = make_float3(pb.x, pb.y, pb.z);
		const float3 n1 = make_float3(oa.x, oa.y, oa.z), n2 = make_float3(ob.x, ob.y, ob.z);
		float a = 1.0f;
		if (acfH)
		{
			a = __ldg(acfH + bin);
		}
		else if (muImg)
		{
			float acc = 0.f;
			auto visit = [&](int o, float w) { acc += w * __ldg(muImg + o); };
			const float3 mo = make_float3(mu.offx, mu.offy, mu.offz);
			siddonWalk<false, false>(mu, f3sub(p1, mo), f3sub(p2, mo), P.tof, 0.f, visit);
			a = expf(-acc * 0.1f);
		}
		const float3 off = make_float3(P.g.offx, P.g.offy, P.g.offz);
		p1 = f3sub(p1, off);
		p2 = f3sub(p2, off);
		float v = a * s;
		float mw = 0.f;
		if constexpr (EM)
		{
			float u;
			if constexpr (MODE == H_BOUND)
				u = forwardEvent<KIND, false, COMP, true>(P, img, p1, p2, n1, n2,
				                                          0.f, k, &mw);
			else
				u = groupSum<TPL>(forwardEvent<KIND, false, COMP>(
				    P, img, p1, p2, n1, n2, 0.f, k, nullptr, part, TPL));
			u *= s;
			u *= a;
			u *= globalScale;
			if (addH)
				u += __ldg(addH + bin);
			if (!(fabsf(u) > denomThr))
				break;
			u = m / u;
			u *= s;
			u *= a;
			u *= globalScale;
			v = u;
		}
		else if constexpr (MODE == H_BOUND)
		{
			if (v != 0.f)
				mw = maxWeightEvent<KIND, false, COMP>(P, p1, p2, n1, n2, 0.f, k);
		}
		if constexpr (MODE == H_BOUND)
			bound = fabsf(v) * mw;
		else if constexpr (MODE == H_FIX)
			backwardEvent<KIND, false, COMP, true>(P, nullptr, v, p1, p2, n1, n2,
			                                       0.f, k, F.acc, fixedScale(F));
		else
			backwardEvent<KIND, false, COMP>(P, out, v, p1, p2, n1, n2, 0.f, k, nullptr,
			                                 0.0, part, TPL);
	} while (false);
	if constexpr (MODE == H_BOUND)
		warpMaxInto(maxBits, bound != bound ? __uint_as_float(0x7fffffffu) : bound);
}

// 8-bit value spread to every third bit (Morton interleave).
__device__ __forceinline__ uint32_t spread3(uint32_t v)
{
	v &= 0xffu;
	v = (v | (v << 8)) & 0x0300F00Fu;
	v = (v | (v << 4)) & 0x030C30C3u;
	v = (v | (v << 2)) & 0x09249249u;
	return v;
}

// Spatial LOR key (29 bits): azimuthal sector of the direction (16 or 64
// over [0, pi), direction folded to dx > 0), the sign of its axial component,
// then the Morton code of the TOF kernel centre (the LOR midpoint without TOF)
// on cells of cell mm from the grid's lower corner (256 per axis with 16
// sectors, 128 with 64).  Rays of one warp then start near each other and run
// nearly parallel, so their voxels overlap.
__device__ __forceinline__ uint64_t spatialKey(const KParams& P, float3 p1, float3 p2,
                                               bool tof, float tofv, float cell,
                                               bool fine)
{
	float3 d = f3sub(p2, p1);
	const float L = sqrtf(d.x * d.x + d.y * d.y + d.z * d.z);
	const float ac = (tof && L > 0.f) ? tofCenter(L, tofv) / L : 0.5f;
	const float3 c = make_float3(p1.x + ac * d.x, p1.y + ac * d.y, p1.z + ac * d.z);
	if (d.x < 0.f || (d.x == 0.f && d.y < 0.f))
		d = make_float3(-d.x, -d.y, -d.z);
	const float phi = atan2f(d.y, d.x);  // (-pi/2, pi/2]
	const uint32_t ns = fine ? 64u : 16u;
	const uint32_t sector = min(ns - 1u, static_cast<uint32_t>(fmaxf(
	                                         0.f, (phi + 1.5707964f) * (static_cast<float>(ns) * 0.31830989f))));
	const uint32_t up = d.z >= 0.f ? 1u : 0u;
	const float top = fine ? 127.f : 255.f;
	auto cellOf = [&](float q, float len) -> uint32_t
	{
		const float u = (q + 0.5f * len) / cell;
		return u <= 0.f ? 0u : (u >= top ? static_cast<uint32_t>(top) : static_cast<uint32_t>(u));
	};
	const uint32_t m = spread3(cellOf(c.x, P.g.lx)) | (spread3(cellOf(c.y, P.g.ly)) << 1) |
	                   (spread3(cellOf(c.z, P.g.lz)) << 2);
	// 16 sectors: sector | up | 24-bit Morton; 64 sectors: sector | up | 21-bit Morton.
	return fine ? (static_cast<uint64_t>(sector) << 22) | (static_cast<uint64_t>(up) << 21) | m
	            : (static_cast<uint64_t>(sector) << 25) | (static_cast<uint64_t>(up) << 24) | m;
}

// Sort key of event e.  Without dynamic frames: subset (e mod S) in bits
// 48..63, ray length bucket (voxel crossings >> bucketShift, at most 127, when
// counts are given) in bits 41..47, LOR key in bits 8..40, TOF in 16 ps steps
// in bits 0..7.  With dynamic frames: subset in bits 52..63, frame in 44..51,
// bucket in 37..43, LOR key in 8..36.  The LOR key is the Histogram3D bin (or
// the ordered detector pair) >> lorShift, or the spatial key.  Grouping rays
// of similar length keeps the threads of a warp iterating together; the LOR
// key keeps neighbouring rays together.
// Sort keys of the event order; vals[e] = e (vals32 when the indices fit 32
// bits, else vals64).  The spatial orders' key already holds the TOF kernel
// centre, so they carry no separate TOF field (8 key bits, one radix pass
// fewer).
__global__ void k_order_keys(KParams P, H3Dev H, bool hasH3, Events E, uint64_t n,
                             uint64_t numSubsets, uint64_t first,
                             const uint32_t* __restrict__ counts,
                             int bucketShift, int lorShift, int spatial, float cell,
                             unsigned long long* __restrict__ keys,
                             unsigned long long* __restrict__ vals64,
                             uint32_t* __restrict__ vals32)
{
	const uint64_t nthreads = static_cast<uint64_t>(gridDim.x) * blockDim.x;
	for (uint64_t e = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	     e < n; e += nthreads)
	{
		uint64_t lorKey = 0;
		const float tofv = E.tof != nullptr ? __ldg(E.tof + e) : 0.f;
		if (spatial)
		{
			float3 p1, p2, n1, n2;
			if (fetchEvent(P, E, e, p1, p2, n1, n2))
				lorKey = spatialKey(P, p1, p2, E.tof != nullptr, tofv, cell, spatial == 2);
		}
		else if (E.d1 != nullptr)
		{
			const uint32_t a = __ldg(E.d1 + e), b = __ldg(E.d2 + e);
			uint64_t bin;
			if (hasH3 && h3Bin(H, a, b, bin))
				lorKey = bin;
			else
				lorKey = static_cast<uint64_t>(min(a, b)) * H.numDets + max(a, b);
			lorKey >>= lorShift;
		}
		uint64_t q = 128;
		if (E.tof != nullptr)
		{
			const float t = tofv / 16.0f + 128.0f;
			q = t <= 0.f ? 0 : (t >= 255.f ? 255 : static_cast<uint64_t>(t));
		}
		const uint64_t bucket = counts ? min(__ldg(counts + e) >> bucketShift, 127u) : 0u;
		uint64_t key;
		if (E.frame != nullptr)
		{
			// Dynamic data: frame after subset, so that one frame's image
			// is traced at a time and stays L2 resident.
			const int f = __ldg(E.frame + e);
			const uint64_t fk = f < 0 ? 255u : static_cast<uint64_t>(min(f, 254));
			key = (((first + e) % numSubsets) << 52) | (fk << 44) | (bucket << 37) |
			      ((lorKey & 0x1FFFFFFFULL) << 8) | q;
		}
		else
		{
			key = (((first + e) % numSubsets) << 48) | (bucket << 41) |
			      ((lorKey & 0x1FFFFFFFFULL) << 8) | q;
		}
		keys[e] = spatial ? (key >> 8) : key;
		if (vals32)
			vals32[e] = static_cast<uint32_t>(e);
		else
			vals64[e] = e;
	}
}

// out[i] = in[i] as 64-bit values.
__global__ void k_widen_u32(const uint32_t* __restrict__ in, uint64_t n,
                            unsigned long long* __restrict__ out)
{
	const uint64_t nthreads = static_cast<uint64_t>(gridDim.x) * blockDim.x;
	for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
	     i += nthreads)
		out[i] = __ldg(in + i);
}

// perm[i] = i * stride (the events of one interleaved subset).
__global__ void k_iota_stride(unsigned long long* __restrict__ perm, uint64_t n,
                              uint64_t stride)
{
	const uint64_t nthreads = static_cast<uint64_t>(gridDim.x) * blockDim.x;
	for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	     i < n; i += nthreads)
		perm[i] = i * stride;
}

// All 32-bit event arrays of a permutation in one pass: one perm read per
// event and up to nine independent loads in flight per thread.
struct GatherSet
{
	const uint32_t* src[9];
	uint32_t* dst[9];
	int count;
};

__global__ void k_gather_set(GatherSet G, const unsigned long long* __restrict__ perm,
                             uint64_t n)
{
	const uint64_t nthreads = static_cast<uint64_t>(gridDim.x) * blockDim.x;
	for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	     i < n; i += nthreads)
	{
		const unsigned long long p = __ldg(perm + i);
		uint32_t v[9];
#pragma unroll
		for (int a = 0; a < 9; a++)
			if (a < G.count)
				v[a] = __ldg(G.src[a] + p);
#pragma unroll
		for (int a = 0; a < 9; a++)
			if (a < G.count)
				G.dst[a][i] = v[a];
	}
}

// Up to four 32-bit arrays interleaved into one 16-byte record per event
// (a streaming pass), so that the permutation then reads one sector per event
// instead of one per array.
__global__ void k_pack4(GatherSet G, int first, int count, uint64_t n,
                        uint4* __restrict__ packed)
{
	const uint64_t nthreads = static_cast<uint64_t>(gridDim.x) * blockDim.x;
	for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	     i < n; i += nthreads)
	{
		uint32_t v[4] = {0u, 0u, 0u, 0u};
#pragma unroll
		for (int a = 0; a < 4; a++)
			if (a < count)
				v[a] = __ldg(G.src[first + a] + i);
		packed[i] = make_uint4(v[0], v[1], v[2], v[3]);
	}
}

__global__ void k_unpack4_gather(GatherSet G, int first, int count, uint64_t n,
                                 const uint4* __restrict__ packed,
                                 const unsigned long long* __restrict__ perm)
{
	const uint64_t nthreads = static_cast<uint64_t>(gridDim.x) * blockDim.x;
	for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	     i < n; i += nthreads)
	{
		const uint4 r = __ldg(packed + __ldg(perm + i));
		const uint32_t v[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
		for (int a = 0; a < 4; a++)
			if (a < count)
				G.dst[first + a][i] = v[a];
	}
}

template <typename T>
__global__ void k_gather(const T* __restrict__ in, const unsigned long long* __restrict__ perm,
                         uint64_t n, int width, T* __restrict__ out)
{
	const uint64_t nthreads = static_cast<uint64_t>(gridDim.x) * blockDim.x;
	for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	     i < n * width; i += nthreads)
	{
		const uint64_t r = i / width, c = i % width;
		out[i] = __ldg(in + perm[r] * width + c);
	}
}

__global__ void k_multiray_offsets(uint64_t count, int numRays,
                                   float* __restrict__ out)
{
	// One item per thread: a warp's threads stay converged across items
	// (a grid-stride loop lets them drift apart between items).
	const uint64_t k = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	const int per = 4 * (numRays - 1);
	if (k < count)
	{
		MultiRay mr;
		mr.init(k, make_float3(1.f, 0.f, 0.f), make_float3(1.f, 0.f, 0.f));
		for (int r = 1; r < numRays; r++)
		{
			float u[4];
			mr.next(u);
			for (int i = 0; i < 4; i++)
				out[k * per + 4 * (r - 1) + i] = u[i];
		}
	}
}

// List-mode records (ListModeLUT file layout: u32 timestamp, u32 d1, u32 d2,
// [f32 TOF], [f32 randoms]) -> structure of arrays.  The lowest index of an
// event with an invalid detector id is recorded in *firstBad.
__global__ void k_unpack_listmode(const uint32_t* __restrict__ raw, uint64_t n,
                                  int fields, int hasTof, int hasRandoms,
                                  uint32_t numDets, uint32_t* __restrict__ ts,
                                  uint32_t* __restrict__ d1,
                                  uint32_t* __restrict__ d2,
                                  float* __restrict__ tof,
                                  float* __restrict__ randoms,
                                  unsigned long long* firstBad)
{
	const uint64_t nthreads = static_cast<uint64_t>(gridDim.x) * blockDim.x;
	for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	     i < n; i += nthreads)
	{
		const uint32_t* r = raw + i * fields;
		const uint32_t a = __ldg(r + 1), b = __ldg(r + 2);
		if (a >= numDets || b >= numDets)
			atomicMin(firstBad, static_cast<unsigned long long>(i));
		if (ts)
			ts[i] = __ldg(r);
		d1[i] = a;
		d2[i] = b;
		int f = 3;
		if (hasTof)
		{
			const float v = __uint_as_float(__ldg(r + f));
			if (tof)
				tof[i] = v;
			f++;
		}
		if (hasRandoms && randoms)
			randoms[i] = __uint_as_float(__ldg(r + f));
	}
}

__global__ void k_lm_to_histo(H3Dev H, const uint32_t* __restrict__ d1,
                              const uint32_t* __restrict__ d2,
                              const float* __restrict__ vals, uint64_t n,
                              float* __restrict__ histo,
                              unsigned long long* invalid)
{
	const uint64_t nthreads = static_cast<uint64_t>(gridDim.x) * blockDim.x;
	for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	     i < n; i += nthreads)
	{
		const float v = vals ? __ldg(vals + i) : 1.0f;
		if (!(v > 0.f))
			continue;
		const uint32_t a = __ldg(d1 + i), b = __ldg(d2 + i);
		if (a == b)
			continue;
		uint64_t bin;
		if (!h3Bin(H, a, b, bin))
		{
			atomicAdd(invalid, 1ULL);
			continue;
		}
		atomicAdd(histo + bin, v);
	}
}

__global__ void k_bins(H3Dev H, const uint32_t* __restrict__ d1,
                       const uint32_t* __restrict__ d2, uint64_t n,
                       uint64_t* __restrict__ bins)
{
	const uint64_t nthreads = static_cast<uint64_t>(gridDim.x) * blockDim.x;
	for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	     i < n; i += nthreads)
	{
		uint64_t b;
		bins[i] = h3Bin(H, __ldg(d1 + i), __ldg(d2 + i), b) ? b : ~0ULL;
	}
}

__global__ void k_pairs(H3Dev H, const uint64_t* __restrict__ bins, uint64_t n,
                        uint32_t* __restrict__ d1, uint32_t* __restrict__ d2)
{
	const uint64_t nthreads = static_cast<uint64_t>(gridDim.x) * blockDim.x;
	const uint64_t total = H.numZBin * H.numPhi * H.numR;
	for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	     i < n; i += nthreads)
	{
		const uint64_t b = __ldg(bins + i);
		uint32_t a = 0, c = 0;
		if (b < total)
			h3Pair(H, b, a, c);
		d1[i] = a;
		d2[i] = c;
	}
}

// ---------------------------------------------------- image-space ops ----
// One thread per voxel of a frame, frames in an inner loop: the broadcast
// sensitivity value is read once per voxel and no index is divided.
__global__ void k_em_update(float* __restrict__ x, const float* __restrict__ u,
                            const float* __restrict__ s, uint64_t J, int64_t nt,
                            int64_t sens_nt, float thr,
                            const float* __restrict__ scale)
{
	const uint64_t nthreads = static_cast<uint64_t>(gridDim.x) * blockDim.x;
	const bool perFrameSens = !scale && sens_nt == nt && nt > 1;
	for (uint64_t j = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < J;
	     j += nthreads)
	{
		const float s0 = __ldg(s + j);
		for (int64_t r = 0; r < nt; r++)
		{
			const uint64_t i = static_cast<uint64_t>(r) * J + j;
			if (perFrameSens)
			{
				const float sv = __ldg(s + i);
				if (sv > thr)
					x[i] *= __ldg(u + i) / sv;
			}
			else if (!scale)
			{
				if (s0 > thr)
					x[i] *= __ldg(u + i) / s0;
			}
			else
			{
				// updateEMThresholdDynamicWithScaling (Image.cpp:760-800).
				const float inv_c = 1.0f / __ldg(scale + r);
				const float thr_r = thr * inv_c;
				if (s0 > thr_r)
					x[i] *= (__ldg(u + i) * inv_c) / s0;
			}
		}
	}
}

// Float4 form of k_em_update (J a multiple of 4; x, u, s 16-byte aligned):
// each thread updates 4 consecutive voxels of every frame with 16-byte
// accesses, several frames unrolled so that their loads are in flight
// together.  The FP32 operations per voxel are those of k_em_update.
__device__ __forceinline__ float emVoxel(float x, float u, float s, float thr,
                                         bool scaled, float inv_c)
{
	if (scaled)
		return s > thr ? x * ((u * inv_c) / s) : x;
	return s > thr ? x * (u / s) : x;
}

__global__ void __launch_bounds__(kBlock)
    k_em_update4(float4* __restrict__ x, const float4* __restrict__ u,
                 const float4* __restrict__ s, uint64_t J4, int64_t nt,
                 int64_t sens_nt, float thr, const float* __restrict__ scale)
{
	const uint64_t nthreads = static_cast<uint64_t>(gridDim.x) * blockDim.x;
	const bool perFrameSens = !scale && sens_nt == nt && nt > 1;
	const bool scaled = scale != nullptr;
	for (uint64_t j = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < J4;
	     j += nthreads)
	{
		const float4 s0 = __ldg(s + j);
		// A group outside the mask in every frame is left untouched (no
		// loads or stores), as the scalar form touches only voxels with s > thr.
		if (!perFrameSens && !scaled &&
		    !(s0.x > thr || s0.y > thr || s0.z > thr || s0.w > thr))
			continue;
#pragma unroll 4
		for (int64_t r = 0; r < nt; r++)
		{
			const uint64_t i = static_cast<uint64_t>(r) * J4 + j;
			const float4 uv = __ldg(u + i);
			const float4 sv = perFrameSens ? __ldg(s + i) : s0;
			float inv_c = 1.f, tr = thr;
			if (scaled)
			{
				// updateEMThresholdDynamicWithScaling (Image.cpp:760-800).
				inv_c = 1.0f / __ldg(scale + r);
				tr = thr * inv_c;
			}
			float4 xv = x[i];
			xv.x = emVoxel(xv.x, uv.x, sv.x, tr, scaled, inv_c);
			xv.y = emVoxel(xv.y, uv.y, sv.y, tr, scaled, inv_c);
			xv.z = emVoxel(xv.z, uv.z, sv.z, tr, scaled, inv_c);
			xv.w = emVoxel(xv.w, uv.w, sv.w, tr, scaled, inv_c);
			x[i] = xv;
		}
	}
}

__global__ void k_threshold(float* __restrict__ x, const float* __restrict__ m,
                            uint64_t J, int64_t nt, int broadcast, float thr,
                            float les, float leo, float gts, float gto)
{
	const uint64_t total = J * static_cast<uint64_t>(nt);
	const uint64_t nthreads = static_cast<uint64_t>(gridDim.x) * blockDim.x;
	for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	     i < total; i += nthreads)
	{
		const float mv = __ldg(m + (broadcast ? i % J : i));
		x[i] = (mv <= thr) ? x[i] * les + leo : x[i] * gts + gto;
	}
}

// Float4 form of k_threshold (J a multiple of 4; x, m 16-byte aligned): 4
// consecutive voxels per thread, frames in an inner loop so that a broadcast
// mask is read once per voxel group and no index is divided.
__device__ __forceinline__ float thrVoxel(float x, float m, float thr, float les,
                                          float leo, float gts, float gto)
{
	return (m <= thr) ? x * les + leo : x * gts + gto;
}

__global__ void __launch_bounds__(kBlock)
    k_threshold4(float4* __restrict__ x, const float4* __restrict__ m,
                 uint64_t J4, int64_t nt, int broadcast, float thr, float les,
                 float leo, float gts, float gto)
{
	const uint64_t nthreads = static_cast<uint64_t>(gridDim.x) * blockDim.x;
	for (uint64_t j = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < J4;
	     j += nthreads)
	{
		const float4 m0 = __ldg(m + j);
#pragma unroll 4
		for (int64_t r = 0; r < nt; r++)
		{
			const uint64_t i = static_cast<uint64_t>(r) * J4 + j;
			const float4 mv = broadcast ? m0 : __ldg(m + i);
			float4 xv = x[i];
			xv.x = thrVoxel(xv.x, mv.x, thr, les, leo, gts, gto);
			xv.y = thrVoxel(xv.y, mv.y, thr, les, leo, gts, gto);
			xv.z = thrVoxel(xv.z, mv.z, thr, les, leo, gts, gto);
			xv.w = thrVoxel(xv.w, mv.w, thr, les, leo, gts, gto);
			x[i] = xv;
		}
	}
}

// Row-major <-> 4 x 2 tiles (tileOffset), one voxel per thread in row-major
// order: the row-major side is read or written coalesced, the tiled side
// within the same 32-byte sectors.
template <bool TO_TILES>
__global__ void k_convert_layout(const float* __restrict__ src, float* __restrict__ dst,
                                 int nx, int ny, int nz, uint64_t total)
{
	const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	if (i >= total)
		return;
	const int nxy = nx * ny;
	const uint64_t nvox = static_cast<uint64_t>(nxy) * nz;
	const uint64_t frame = i / nvox;
	const int r = static_cast<int>(i - frame * nvox);
	const int z = r / nxy;
	const int xy = r - z * nxy;
	const int y = xy / nx;
	const int x = xy - y * nx;
	const uint64_t t = frame * nvox + static_cast<uint64_t>(tileOffset(x, y, z, nx, nxy));
	if constexpr (TO_TILES)
		dst[t] = __ldg(src + i);
	else
		dst[i] = __ldg(src + t);
}

__global__ void k_fill(float* __restrict__ x, uint64_t n, float v)
{
	const uint64_t nthreads = static_cast<uint64_t>(gridDim.x) * blockDim.x;
	for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	     i < n; i += nthreads)
		x[i] = v;
}

__global__ void k_scale(float* __restrict__ x, uint64_t n, float v)
{
	const uint64_t nthreads = static_cast<uint64_t>(gridDim.x) * blockDim.x;
	for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	     i < n; i += nthreads)
		x[i] *= v;
}

// One pass of the separable image-space PSF along AXIS (0 x, 1 y, 2 z):
// dst[i] = sum_kk k[kk + c] * src[circ(i - kk)], kk = -c..c, circular border,
// FP32 sums in tap order (OperatorPsf::convolve, src/operators/OperatorPsf.cpp:288-375).
// Blocks of kPsfBX x kPsfBY threads cover an (x, y) tile; each thread takes
// kPsfPlanes consecutive (z, frame) planes at a time, so every tap issues
// kPsfPlanes independent loads, and no thread divides a 64-bit index.  A warp
// reads 32 consecutive x for every tap (coalesced along every axis).
// NK > 0 fixes the number of taps at compile time (the tap loop unrolls and
// all loads of a plane group are in flight together); NK = 0 reads nk.
constexpr int kPsfBX = 32, kPsfBY = 8, kPsfPlanes = 4;
template <int AXIS, int NK>
__global__ void __launch_bounds__(kPsfBX * kPsfBY)
k_psf_pass(const float* __restrict__ src, float* __restrict__ dst, int nx, int ny, int nz,
           int planes, const float* __restrict__ k, int nkRuntime)
{
	const int nk = NK > 0 ? NK : nkRuntime;
	const int x = blockIdx.x * kPsfBX + threadIdx.x;
	const int y = blockIdx.y * kPsfBY + threadIdx.y;
	if (x >= nx || y >= ny)
		return;
	const int c = nk / 2;
	const int n = AXIS == 0 ? nx : (AXIS == 1 ? ny : nz);
	const int64_t plane = static_cast<int64_t>(nx) * ny;
	const int64_t stride = AXIS == 0 ? 1 : (AXIS == 1 ? nx : plane);
	for (int zt0 = blockIdx.z * kPsfPlanes; zt0 < planes; zt0 += gridDim.z * kPsfPlanes)
	{
		const float* base[kPsfPlanes];
		int coord[kPsfPlanes];
		float sum[kPsfPlanes];
#pragma unroll
		for (int q = 0; q < kPsfPlanes; q++)
		{
			// Past the last plane, repeat it (loads stay in bounds, no store).
			const int zt = min(zt0 + q, planes - 1);
			const int64_t i = zt * plane + static_cast<int64_t>(y) * nx + x;
			coord[q] = AXIS == 0 ? x : (AXIS == 1 ? y : zt % nz);
			base[q] = src + (i - coord[q] * stride);
			sum[q] = 0.f;
		}
#pragma unroll
		for (int kk = -c; kk <= c; kk++)
		{
			const float tap = __ldg(k + kk + c);
#pragma unroll
			for (int q = 0; q < kPsfPlanes; q++)
			{
				int r = coord[q] - kk;
				r = r < 0 ? r + n : (r >= n ? r - n : r);
				// Rounded product and sum, no contraction into an FMA: the
				// reference operator multiplies and adds separately.
				sum[q] = __fadd_rn(sum[q], __fmul_rn(tap, __ldg(base[q] + r * stride)));
			}
		}
#pragma unroll
		for (int q = 0; q < kPsfPlanes; q++)
			if (zt0 + q < planes)
				dst[(zt0 + q) * plane + static_cast<int64_t>(y) * nx + x] = sum[q];
	}
}

// Vector form of k_psf_pass for rows of a multiple of 4 voxels (16-byte
// aligned images): each thread produces 4 consecutive x of kPsfPlanes planes
// with 16-byte loads.  Along y and z every tap is one float4 load; along x the
// thread loads the 2D+1 aligned chunks around its own (circular chunk index,
// which wraps by whole periods because nx is a multiple of 4) and slides the
// taps over them in registers.  Same products and sums in the same order as
// the scalar form, so the results are bit-identical.
template <int AXIS, int NK>
__global__ void __launch_bounds__(kPsfBX * kPsfBY)
k_psf_pass4(const float* __restrict__ src, float* __restrict__ dst, int nx, int ny, int nz,
            int planes, const float* __restrict__ k)
{
	constexpr int C = NK / 2;
	constexpr int D = (C + 3) / 4;
	const int nxc = nx >> 2;
	const int jx = blockIdx.x * kPsfBX + threadIdx.x;
	const int y = blockIdx.y * kPsfBY + threadIdx.y;
	if (jx >= nxc || y >= ny)
		return;
	float taps[NK];
#pragma unroll
	for (int i = 0; i < NK; i++)
		taps[i] = __ldg(k + i);
	const int64_t plane = static_cast<int64_t>(nx) * ny;
	for (int zt0 = blockIdx.z * kPsfPlanes; zt0 < planes; zt0 += gridDim.z * kPsfPlanes)
	{
		float4 acc[kPsfPlanes];
#pragma unroll
		for (int q = 0; q < kPsfPlanes; q++)
		{
			const int zt = min(zt0 + q, planes - 1);
			const float* row = src + zt * plane + static_cast<int64_t>(y) * nx;
			float out[4];
			if constexpr (AXIS == 0)
			{
				float w[4 * (2 * D + 1)];
#pragma unroll
				for (int d = -D; d <= D; d++)
				{
					int j = jx + d;
					j = j < 0 ? j + nxc : (j >= nxc ? j - nxc : j);
					const float4 v = __ldg(reinterpret_cast<const float4*>(row) + j);
					w[4 * (d + D) + 0] = v.x;
					w[4 * (d + D) + 1] = v.y;
					w[4 * (d + D) + 2] = v.z;
					w[4 * (d + D) + 3] = v.w;
				}
#pragma unroll
				for (int m = 0; m < 4; m++)
				{
					float sum = 0.f;
#pragma unroll
					for (int kk = -C; kk <= C; kk++)
						sum = __fadd_rn(sum, __fmul_rn(taps[kk + C], w[4 * D + m - kk]));
					out[m] = sum;
				}
			}
			else
			{
				const int n = AXIS == 1 ? ny : nz;
				const int coord = AXIS == 1 ? y : zt % nz;
				const int64_t stride = AXIS == 1 ? nx : plane;
				const float* col = row - coord * stride + 4 * jx;
				out[0] = out[1] = out[2] = out[3] = 0.f;
#pragma unroll
				for (int kk = -C; kk <= C; kk++)
				{
					int r = coord - kk;
					r = r < 0 ? r + n : (r >= n ? r - n : r);
					const float4 v = __ldg(reinterpret_cast<const float4*>(col + r * stride));
					const float t = taps[kk + C];
					out[0] = __fadd_rn(out[0], __fmul_rn(t, v.x));
					out[1] = __fadd_rn(out[1], __fmul_rn(t, v.y));
					out[2] = __fadd_rn(out[2], __fmul_rn(t, v.z));
					out[3] = __fadd_rn(out[3], __fmul_rn(t, v.w));
				}
			}
			acc[q] = make_float4(out[0], out[1], out[2], out[3]);
		}
#pragma unroll
		for (int q = 0; q < kPsfPlanes; q++)
			if (zt0 + q < planes)
				*reinterpret_cast<float4*>(dst + (zt0 + q) * plane +
				                           static_cast<int64_t>(y) * nx + 4 * jx) = acc[q];
	}
}

// Kernel sizes up to 15 taps run the unrolled instantiation.
// vec: rows of a multiple of 4 voxels and 16-byte aligned buffers; grid.x
// then counts chunks of 4 x.
template <int AXIS>
void psfPass(dim3 grid, dim3 block, cudaStream_t st, const float* src, float* dst,
             const int* dims, int planes, const float* k, int nk, bool vec)
{
	dim3 grid4 = grid;
	grid4.x = (dims[0] / 4 + kPsfBX - 1) / kPsfBX;
#define YRTB_PSF_CASE(N)                                                                  \
	case N:                                                                               \
		if (vec)                                                                          \
			k_psf_pass4<AXIS, N><<<grid4, block, 0, st>>>(src, dst, dims[0], dims[1],     \
			                                              dims[2], planes, k);            \
		else                                                                              \
			k_psf_pass<AXIS, N><<<grid, block, 0, st>>>(src, dst, dims[0], dims[1],       \
			                                            dims[2], planes, k, nk);          \
		return;
	switch (nk)
	{
		YRTB_PSF_CASE(1)
		YRTB_PSF_CASE(3)
		YRTB_PSF_CASE(5)
		YRTB_PSF_CASE(7)
		YRTB_PSF_CASE(9)
		YRTB_PSF_CASE(11)
		YRTB_PSF_CASE(13)
		YRTB_PSF_CASE(15)
	default:
		k_psf_pass<AXIS, 0><<<grid, block, 0, st>>>(src, dst, dims[0], dims[1], dims[2],
		                                            planes, k, nk);
	}
#undef YRTB_PSF_CASE
}

// ------------------------------------------- spatially variant image PSF --
// OperatorVarPsf (src/operators/OperatorVarPsf.cpp:290-455): every voxel has
// its own 3-D kernel, the LUT entry nearest to |voxel centre - image centre|
// (x, y, z gaps, clamped at the LUT's range).
struct VarPsfDev
{
	const float* w;     // all kernels' weights, z-major, then y, then x
	const int4* meta;   // per kernel: offset into w, half sizes x, y, z
	int lutX, lutY, lutZ;
	float gapX, gapY, gapZ;
	float vx, vy, vz;
	float cx, cy, cz;   // image centre: n * v / 2 in FP32
	int maxHx, maxHy, maxHz;
};

// LUT coordinate of index i along one axis (OperatorVarPsf::findNearestKernel
// with the distances of varconvolve: |(i + 0.5) v - centre| in FP64, then
// FP32, divided by the gap, rounded, clamped).  The LUT index of voxel
// (i, j, k) is a(i) + A (b(j) + B c(k)): separable, so each block tabulates
// the three axes once in shared memory.
__device__ __forceinline__ int varPsfAxis(int i, float v, float centre, float gap, int dim)
{
	const float t = static_cast<float>(fabs((i + 0.5) * static_cast<double>(v) - centre));
	const int a = static_cast<int>(roundf(fabsf(t) / gap));
	return a >= dim ? dim - 1 : a;
}

__device__ __forceinline__ int circ1(int n, int x)
{
	return x < 0 ? x + n : (x >= n ? x - n : x);
}

// Forward (applyA): out[p] = sum over the kernel of p of in[p + d] w_p(d),
// d in z, y, x order, FP32 products and sums as the reference's loop.
// Adjoint (applyAH): the reference scatters in[q] w_q(d) to q + d; here each
// output gathers out[p] = sum_d in[p - d] w_{p-d}(d) over the largest kernel
// support (no atomics; the FP32 sum order differs from the scatter's).
template <bool ADJ>
__global__ void __launch_bounds__(kPsfBX * kPsfBY)
k_varpsf(const float* __restrict__ src, float* __restrict__ dst, int nx, int ny, int nz,
         int planes, VarPsfDev P)
{
	extern __shared__ int varAxis[];  // nx + ny + nz: LUT offsets per axis
	int* ax = varAxis;
	int* ay = ax + nx;
	int* az = ay + ny;
	for (int t = threadIdx.y * kPsfBX + threadIdx.x; t < nx + ny + nz; t += kPsfBX * kPsfBY)
	{
		if (t < nx)
			ax[t] = varPsfAxis(t, P.vx, P.cx, P.gapX, P.lutX);
		else if (t < nx + ny)
			ay[t - nx] = P.lutX * varPsfAxis(t - nx, P.vy, P.cy, P.gapY, P.lutY);
		else
			az[t - nx - ny] =
			    P.lutX * P.lutY * varPsfAxis(t - nx - ny, P.vz, P.cz, P.gapZ, P.lutZ);
	}
	__syncthreads();
	const int x = blockIdx.x * kPsfBX + threadIdx.x;
	const int y = blockIdx.y * kPsfBY + threadIdx.y;
	if (x >= nx || y >= ny)
		return;
	const int64_t plane = static_cast<int64_t>(nx) * ny;
	for (int zt = blockIdx.z; zt < planes; zt += gridDim.z)
	{
		const int z = zt % nz;
		const float* frame = src + (zt - z) * plane;
		float sum = 0.f;
		if (!ADJ)
		{
			const int4 m = __ldg(P.meta + ax[x] + ay[y] + az[z]);
			const float* w = P.w + m.x;
			for (int dz = -m.w; dz <= m.w; dz++)
			{
				const float* pz = frame + circ1(nz, z + dz) * plane;
				for (int dy = -m.z; dy <= m.z; dy++)
				{
					const float* py = pz + static_cast<int64_t>(circ1(ny, y + dy)) * nx;
					for (int dx = -m.y; dx <= m.y; dx++, w++)
						sum = __fadd_rn(sum, __fmul_rn(__ldg(py + circ1(nx, x + dx)), __ldg(w)));
				}
			}
		}
		else
		{
			for (int dz = -P.maxHz; dz <= P.maxHz; dz++)
			{
				const int qz = circ1(nz, z - dz);
				const int cz = az[qz];
				for (int dy = -P.maxHy; dy <= P.maxHy; dy++)
				{
					const int qy = circ1(ny, y - dy);
					const int cyz = cz + ay[qy];
					for (int dx = -P.maxHx; dx <= P.maxHx; dx++)
					{
						const int qx = circ1(nx, x - dx);
						const int4 m = __ldg(P.meta + cyz + ax[qx]);
						if (dx < -m.y || dx > m.y || dy < -m.z || dy > m.z || dz < -m.w ||
						    dz > m.w)
							continue;
						const int tap = ((dz + m.w) * (2 * m.z + 1) + (dy + m.z)) * (2 * m.y + 1) +
						                (dx + m.y);
						sum = __fadd_rn(sum, __fmul_rn(__ldg(frame + qz * plane +
						                                     static_cast<int64_t>(qy) * nx + qx),
						                               __ldg(P.w + m.x + tap)));
					}
				}
			}
		}
		dst[static_cast<int64_t>(zt) * plane + static_cast<int64_t>(y) * nx + x] = sum;
	}
}

// ------------------------------------------------- low-rank dynamic image --
// Frame t of a low-rank image is x_t = sum_l H[l][t] W_l (W: rank images, H:
// rank x frames basis), the ProjectorUpdaterLR / ProjectorUpdaterDeviceLR
// model (src/operators/ProjectorUpdater.cpp:228-280,
// include/yrt-pet/operators/ProjectorUpdaterDevice.cuh:53-225).  The reference
// applies the rank sum at every voxel crossing (rank gathers forward, rank
// atomics backward).  Here the frames are expanded once per subset, the
// frame-indexed projection kernels run on them (one gather / one atomic per
// crossing), and the frame-indexed EM image is contracted back onto W or H.
constexpr int kLrMaxRank = 32;
constexpr int kLrTile = 128;      // voxels per shared-memory tile (H contraction)
constexpr int kLrPairs = 8;       // (rank, frame) pairs per thread, 256 threads
constexpr int kLrBlock = 256;

// X[t][j] = sum_l W[l][j] * H[l][t], l ascending, rounded products and sums
// (the CPU updater's forwardUpdate order).
template <int RMAX>
__global__ void __launch_bounds__(kBlock)
k_lr_expand(const float* __restrict__ W, const float* __restrict__ H, int R, int T, uint64_t J,
            float* __restrict__ X)
{
	const uint64_t nthreads = static_cast<uint64_t>(gridDim.x) * blockDim.x;
	for (uint64_t j = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < J;
	     j += nthreads)
	{
		float w[RMAX];
#pragma unroll
		for (int l = 0; l < RMAX; l++)
			w[l] = l < R ? __ldg(W + l * J + j) : 0.f;
		for (int t = 0; t < T; t++)
		{
			float x = 0.f;
#pragma unroll
			for (int l = 0; l < RMAX; l++)
				if (l < R)
					x = __fadd_rn(x, __fmul_rn(w[l], __ldg(H + l * T + t)));
			X[static_cast<uint64_t>(t) * J + j] = x;
		}
	}
}

// Wn[l][j] = sum_t E[t][j] * H[l][t], t ascending.
template <int RMAX>
__global__ void __launch_bounds__(kBlock)
k_lr_contract_w(const float* __restrict__ E, const float* __restrict__ H, int R, int T,
                uint64_t J, float* __restrict__ Wn)
{
	const uint64_t nthreads = static_cast<uint64_t>(gridDim.x) * blockDim.x;
	for (uint64_t j = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < J;
	     j += nthreads)
	{
		float acc[RMAX];
#pragma unroll
		for (int l = 0; l < RMAX; l++)
			acc[l] = 0.f;
		for (int t = 0; t < T; t++)
		{
			const float e = __ldg(E + static_cast<uint64_t>(t) * J + j);
#pragma unroll
			for (int l = 0; l < RMAX; l++)
				if (l < R)
					acc[l] = __fadd_rn(acc[l], __fmul_rn(e, __ldg(H + l * T + t)));
		}
#pragma unroll
		for (int l = 0; l < RMAX; l++)
			if (l < R)
				Wn[l * J + j] = acc[l];
	}
}

// Vector forms of k_lr_expand / k_lr_contract_w for images of a multiple of 4
// voxels (16-byte aligned, rank <= 16): 4 consecutive voxels per thread with
// 16-byte loads and stores, the same products and sums per voxel.
__device__ __forceinline__ float4 lrMulAdd4(float4 acc, float4 v, float h)
{
	acc.x = __fadd_rn(acc.x, __fmul_rn(v.x, h));
	acc.y = __fadd_rn(acc.y, __fmul_rn(v.y, h));
	acc.z = __fadd_rn(acc.z, __fmul_rn(v.z, h));
	acc.w = __fadd_rn(acc.w, __fmul_rn(v.w, h));
	return acc;
}

template <int RMAX>
__global__ void __launch_bounds__(kBlock)
k_lr_expand4(const float4* __restrict__ W, const float* __restrict__ H, int R, int T,
             uint64_t J4, float4* __restrict__ X)
{
	const uint64_t nthreads = static_cast<uint64_t>(gridDim.x) * blockDim.x;
	for (uint64_t j = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < J4;
	     j += nthreads)
	{
		float4 w[RMAX];
#pragma unroll
		for (int l = 0; l < RMAX; l++)
			w[l] = l < R ? __ldg(W + l * J4 + j) : make_float4(0.f, 0.f, 0.f, 0.f);
		for (int t = 0; t < T; t++)
		{
			float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
			for (int l = 0; l < RMAX; l++)
				if (l < R)
					x = lrMulAdd4(x, w[l], __ldg(H + l * T + t));
			X[static_cast<uint64_t>(t) * J4 + j] = x;
		}
	}
}

template <int RMAX>
__global__ void __launch_bounds__(kBlock)
k_lr_contract_w4(const float4* __restrict__ E, const float* __restrict__ H, int R, int T,
                 uint64_t J4, float4* __restrict__ Wn)
{
	const uint64_t nthreads = static_cast<uint64_t>(gridDim.x) * blockDim.x;
	for (uint64_t j = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < J4;
	     j += nthreads)
	{
		float4 acc[RMAX];
#pragma unroll
		for (int l = 0; l < RMAX; l++)
			acc[l] = make_float4(0.f, 0.f, 0.f, 0.f);
		for (int t = 0; t < T; t++)
		{
			const float4 e = __ldg(E + static_cast<uint64_t>(t) * J4 + j);
#pragma unroll
			for (int l = 0; l < RMAX; l++)
				if (l < R)
					acc[l] = lrMulAdd4(acc[l], e, __ldg(H + l * T + t));
		}
#pragma unroll
		for (int l = 0; l < RMAX; l++)
			if (l < R)
				Wn[l * J4 + j] = acc[l];
	}
}

// Split-J contraction: partial[b][l*T + t] = sum over block b's voxels of
// W[l][j] * E[t][j] (rounded FP32 product, FP64 sum).  Tiles of kLrTile voxels
// of every W row and E row sit in shared memory (rows padded to kLrTile + 1
// floats: the 32 threads of a warp read 32 different E rows without bank
// conflicts); each thread owns up to kLrPairs (l, t) pairs.
__global__ void __launch_bounds__(kLrBlock)
k_lr_contract_h(const float* __restrict__ W, const float* __restrict__ E, int R, int T,
                uint64_t J, double* __restrict__ partial)
{
	extern __shared__ float lrTile[];
	constexpr int ld = kLrTile + 1;
	const int P = R * T;
	double acc[kLrPairs];
#pragma unroll
	for (int q = 0; q < kLrPairs; q++)
		acc[q] = 0.0;
	for (uint64_t j0 = static_cast<uint64_t>(blockIdx.x) * kLrTile; j0 < J;
	     j0 += static_cast<uint64_t>(gridDim.x) * kLrTile)
	{
		const uint64_t left = J - j0;
		const int n = left < static_cast<uint64_t>(kLrTile) ? static_cast<int>(left) : kLrTile;
		__syncthreads();
		for (int idx = threadIdx.x; idx < (R + T) * kLrTile; idx += blockDim.x)
		{
			const int row = idx / kLrTile, col = idx - row * kLrTile;
			float v = 0.f;
			if (col < n)
				v = row < R ? __ldg(W + row * J + j0 + col)
				            : __ldg(E + static_cast<uint64_t>(row - R) * J + j0 + col);
			lrTile[row * ld + col] = v;
		}
		__syncthreads();
#pragma unroll
		for (int q = 0; q < kLrPairs; q++)
		{
			const int k = threadIdx.x + q * kLrBlock;
			if (k < P)
			{
				const int l = k / T, t = k - (k / T) * T;
				const float* a = lrTile + l * ld;
				const float* b = lrTile + (R + t) * ld;
				double sum = 0.0;
				for (int i = 0; i < n; i++)
					sum += static_cast<double>(__fmul_rn(a[i], b[i]));
				acc[q] += sum;
			}
		}
	}
#pragma unroll
	for (int q = 0; q < kLrPairs; q++)
	{
		const int k = threadIdx.x + q * kLrBlock;
		if (k < P)
			partial[static_cast<uint64_t>(blockIdx.x) * P + k] = acc[q];
	}
}

// out[k] = sum over blocks b (ascending) of partial[b][k].
__global__ void k_lr_finish(const double* __restrict__ partial, int blocks, int P,
                            double* __restrict__ out)
{
	for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < P; k += gridDim.x * blockDim.x)
	{
		double s = 0.0;
		for (int b = 0; b < blocks; b++)
			s += partial[static_cast<uint64_t>(b) * P + k];
		out[k] = s;
	}
}

// H[r][t] *= float(Hn[r][t]) * (1 / max(cH[r], eps))  (LREM::applyHUpdate,
// src/recon/LREM.cpp:175-199: the numerator is held in FP32 there).
__global__ void k_lr_update_h(float* __restrict__ H, const double* __restrict__ Hn,
                              const float* __restrict__ cH, int R, int T, float eps)
{
	for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < R * T; k += gridDim.x * blockDim.x)
	{
		const int r = k / T;
		const float inv = 1.0f / fmaxf(cH[r], eps);
		H[k] = __fmul_rn(H[k], __fmul_rn(static_cast<float>(Hn[k]), inv));
	}
}

int g_numSMs = 0;

// Blocks for one item per thread.
unsigned gridAll(uint64_t n)
{
	return static_cast<unsigned>(std::max<uint64_t>(1, (n + kBlock - 1) / kBlock));
}

unsigned gridFor(uint64_t n, int perSM = 8)
{
	if (g_numSMs == 0)
	{
		int dev = 0;
		cudaGetDevice(&dev);
		cudaDeviceGetAttribute(&g_numSMs, cudaDevAttrMultiProcessorCount, dev);
		if (g_numSMs <= 0)
			g_numSMs = 148;
	}
	const uint64_t need = (n + kBlock - 1) / kBlock;
	const uint64_t cap = static_cast<uint64_t>(g_numSMs) * perSM;
	return static_cast<unsigned>(std::max<uint64_t>(1, std::min(need, cap)));
}

// Temporaries of the event ordering, the attenuation factors and the
// autotuner come from a stream-ordered pool the library keeps per device,
// with freed blocks retained for later calls (the default pool returns them
// to the CUDA driver at every synchronisation, and re-mapping a gigabyte of
// ordering keys costs more than the sort itself).
constexpr int kMaxPoolDevices = 64;
std::mutex g_poolLock;
cudaMemPool_t g_pools[kMaxPoolDevices] = {};

cudaError_t poolAlloc(void** p, size_t bytes, cudaStream_t st)
{
	constexpr int kMaxDevices = kMaxPoolDevices;
	std::mutex& lock = g_poolLock;
	cudaMemPool_t* pools = g_pools;
	int dev = 0;
	cudaError_t e = cudaGetDevice(&dev);
	if (e != cudaSuccess)
		return e;
	if (dev < 0 || dev >= kMaxDevices)
		return cudaMallocAsync(p, bytes, st);
	{
		std::lock_guard<std::mutex> guard(lock);
		if (pools[dev] == nullptr)
		{
			cudaMemPoolProps props{};
			props.allocType = cudaMemAllocationTypePinned;
			props.location.type = cudaMemLocationTypeDevice;
			props.location.id = dev;
			cudaMemPool_t pool = nullptr;
			if ((e = cudaMemPoolCreate(&pool, &props)) != cudaSuccess)
				return e;
			uint64_t keep = ~uint64_t(0);
			if ((e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep)) !=
			    cudaSuccess)
				return e;
			pools[dev] = pool;
		}
	}
	return cudaMallocFromPoolAsync(p, bytes, pools[dev], st);
}

template <typename T>
cudaError_t poolAlloc(T** p, size_t bytes, cudaStream_t st)
{
	return poolAlloc(reinterpret_cast<void**>(p), bytes, st);
}

Geom makeGeom(const yrtb_image_params& ip)
{
	Geom g{};
	g.nt = static_cast<int>(ip.nt);
	g.nx = static_cast<int>(ip.nx);
	g.ny = static_cast<int>(ip.ny);
	g.nz = static_cast<int>(ip.nz);
	g.nxy = ip.nx * ip.ny;
	g.nvox = ip.nx * ip.ny * ip.nz;
	g.lx = ip.length_x;
	g.ly = ip.length_y;
	g.lz = ip.length_z;
	// ImageParams::completeDimInfo / setup (ImageParams.cpp:205-270).
	g.vx = ip.length_x / static_cast<float>(ip.nx);
	g.vy = ip.length_y / static_cast<float>(ip.ny);
	g.vz = ip.length_z / static_cast<float>(ip.nz);
	float fr = std::max(ip.length_x / 2.0f, ip.length_y / 2.0f);
	fr -= std::max(g.vx, g.vy) / 1000.0f;
	g.fovRadius = fr;
	auto snap = [](float o) { return std::fabs(o) < 1e-4f ? 0.0f : o; };
	g.offx = snap(ip.off_x);
	g.offy = snap(ip.off_y);
	g.offz = snap(ip.off_z);
	return g;
}

bool validImage(const yrtb_image_params* ip)
{
	return ip && ip->nx > 0 && ip->ny > 0 && ip->nz > 0 && ip->nt > 0 &&
	       ip->length_x > 0 && ip->length_y > 0 && ip->length_z > 0 &&
	       ip->nx * ip->ny * ip->nz < (int64_t(1) << 31);
}

}  // namespace

struct yrtb_projector
{
	yrtb_scanner sc;
	yrtb_image_params ip;
	yrtb_projector_params pp;
	KParams P;
	int kind;
	bool hasTof;
	bool comp;
	std::unique_ptr<H3Host> h3;
	H3Dev h3d;
	float4* d_pos = nullptr;
	float4* d_ori = nullptr;
	float* d_taps = nullptr;
	float* d_flipped = nullptr;
	float* d_prefix = nullptr;
	float* d_prefixFlipped = nullptr;
	int32_t* d_ring = nullptr;
	int2* d_z = nullptr;
	unsigned long long* d_err = nullptr;
	// Multi-ray offset table (yrtb_multiray_table): capacity in item indices.
	float* d_mrTable = nullptr;
	uint64_t mrCapacity = 0;
	// Launch configuration of the single-ray Siddon event kernels.
	yrtb_launch_config launch{256, 1, 3, YRTB_ORDER_LOR, 1, 2};
	// Layout of the images of the list-mode projections (YRTB_LAYOUT_*).
	int layout = YRTB_LAYOUT_ROW_MAJOR;
	// Deterministic back projection: fixed-point image (nvox * nt) and bound.
	bool det = false;
	unsigned long long* d_fix = nullptr;
	unsigned* d_fixMax = nullptr;
	int device = 0;

	~yrtb_projector()
	{
		cudaFree(d_fix);
		cudaFree(d_fixMax);
		cudaFree(d_pos);
		cudaFree(d_ori);
		cudaFree(d_taps);
		cudaFree(d_flipped);
		cudaFree(d_prefix);
		cudaFree(d_prefixFlipped);
		cudaFree(d_ring);
		cudaFree(d_z);
		cudaFree(d_err);
		cudaFree(d_mrTable);
	}
};

// Spatially variant image-space PSF: kernel LUT on the device.
struct yrtb_varpsf
{
	float* w = nullptr;
	int4* meta = nullptr;
	int numKernels = 0;
	int lut[3] = {0, 0, 0};
	float gap[3] = {0, 0, 0};
	int maxH[3] = {0, 0, 0};
	int device = 0;
	~yrtb_varpsf()
	{
		cudaFree(w);
		cudaFree(meta);
	}
};

// Separable image-space PSF: kernels and flipped kernels per axis.
struct yrtb_psf
{
	float* k[3] = {nullptr, nullptr, nullptr};
	float* kf[3] = {nullptr, nullptr, nullptr};
	int n[3] = {0, 0, 0};
	int device = 0;
	~yrtb_psf()
	{
		for (int a = 0; a < 3; a++)
		{
			cudaFree(k[a]);
			cudaFree(kf[a]);
		}
	}
};

namespace
{
Events toDev(const yrtb_events* ev)
{
	Events E{};
	E.d1 = ev->d1;
	E.d2 = ev->d2;
	E.lor = ev->lor;
	E.tof = ev->tof_ps;
	E.frame = ev->frame;
	E.mframe = ev->motion_frame;
	E.motion = ev->motion;
	E.numMotion = ev->num_motion_frames;
	E.meas = ev->measurement;
	E.sens = ev->sens;
	E.att = ev->att;
	E.add = ev->additive;
	E.orient = ev->orient;
	return E;
}

// An event set with no events: its per-event arrays (and the caller's
// per-event outputs) may be null, since empty buffers have no storage.
bool emptyEvents(const yrtb_events* ev)
{
	return ev != nullptr && ev->count == 0;
}

yrtb_status checkEvents(const yrtb_projector* h, const yrtb_events* ev,
                        yrtb_range& r, bool needTof)
{
	if (!h || !ev)
		return fail(YRTB_ERR_ARGUMENT, "null projector or events");
	if (ev->count == 0)
	{
		// Nothing to project: accepted whatever arrays are given (an empty
		// tensor has no storage), and the range is empty.
		if (r.stride == 0)
			r.stride = 1;
		r.count = 0;
		return YRTB_OK;
	}
	if (!ev->d1 && !ev->lor)
		return fail(YRTB_ERR_ARGUMENT, "events need detector ids or LORs");
	if ((ev->d1 == nullptr) != (ev->d2 == nullptr))
		return fail(YRTB_ERR_ARGUMENT, "d1 and d2 must both be given");
	if (ev->motion_frame && (!ev->motion || ev->num_motion_frames == 0))
		return fail(YRTB_ERR_ARGUMENT, "motion frames given without transforms");
	if (h->kind != K_SIDDON && !ev->d1 && !ev->orient)
		return fail(YRTB_ERR_ARGUMENT,
		            "distance-driven and multi-ray projection need detector ids "
		            "or, with LORs, crystal orientations");
	if (needTof && h->hasTof && !ev->tof_ps)
		return fail(YRTB_ERR_ARGUMENT, "TOF projector requires per-event TOF values");
	if (r.stride == 0)
		r.stride = 1;
	if (r.start >= ev->count && ev->count > 0)
		return fail(YRTB_ERR_ARGUMENT, "range start beyond the event count");
	const uint64_t avail = ev->count == 0 ? 0 : (ev->count - r.start + r.stride - 1) / r.stride;
	if (r.count == 0 || r.count > avail)
		r.count = avail;
	return YRTB_OK;
}

// Calls fn(kind, tof, comp) with the projector's configuration as
// std::integral_constant / bool_constant values (compensated arithmetic
// exists for the Siddon projectors and, as prefix-sum PSF integrals and
// products with reciprocals of the LOR's and rows' constant denominators, for
// distance-driven projection with a PSF).
template <typename Fn>
void withConfig(const yrtb_projector* h, Fn&& fn)
{
	const bool tof = h->hasTof, comp = h->comp;
	auto go = [&](auto kind)
	{
		using K = decltype(kind);
		if constexpr (K::value == K_SIDDON || K::value == K_SIDDON_MR ||
		              K::value == K_DD_PSF)
		{
			if (tof && comp)
				fn(kind, std::true_type{}, std::true_type{});
			else if (tof)
				fn(kind, std::true_type{}, std::false_type{});
			else if (comp)
				fn(kind, std::false_type{}, std::true_type{});
			else
				fn(kind, std::false_type{}, std::false_type{});
		}
		else
		{
			if (tof)
				fn(kind, std::true_type{}, std::false_type{});
			else
				fn(kind, std::false_type{}, std::false_type{});
		}
	};
	switch (h->kind)
	{
	case K_SIDDON: go(std::integral_constant<int, K_SIDDON>{}); break;
	case K_SIDDON_MR: go(std::integral_constant<int, K_SIDDON_MR>{}); break;
	case K_DD: go(std::integral_constant<int, K_DD>{}); break;
	default: go(std::integral_constant<int, K_DD_PSF>{}); break;
	}
}

// Clears the fixed-point image (frames 0..nt-1) and the bound of a
// deterministic back projection over n items.
yrtb_status fixedBegin(yrtb_projector* h, uint64_t n, cudaStream_t st, Fixed& F)
{
	const uint64_t J = static_cast<uint64_t>(h->P.g.nvox) * h->ip.nt;
	YRTB_CUDA(cudaMemsetAsync(h->d_fix, 0, J * sizeof(unsigned long long), st));
	YRTB_CUDA(cudaMemsetAsync(h->d_fixMax, 0, sizeof(unsigned), st));
	F = Fixed{h->d_fix, h->d_fixMax, n};
	return YRTB_OK;
}

void fixedEnd(yrtb_projector* h, const Fixed& F, float* out, cudaStream_t st)
{
	const uint64_t J = static_cast<uint64_t>(h->P.g.nvox) * h->ip.nt;
	k_fixed_finish<<<gridFor(J, 8), kBlock, 0, st>>>(h->d_fix, J, F, out);
}

// Siddon event kernel with block size B and the projector's threads per LOR:
// pieces of a single ray (compensated arithmetic only; 1 otherwise), or one
// lane per ray of a multi-ray projector.
template <int OP, int K, bool T, bool C, int B, bool TILE = false>
void launchTuned(const yrtb_projector* h, const Events& E, Range R,
                 const float* in, float* out, float gs, float thr,
                 cudaStream_t st, const Fixed& F)
{
	// Float4 groups need 16-byte aligned frames of the images read and
	// written (every frame starts at a multiple of nvox floats).
	const float* img = OP == OP_BWD ? out : in;
	const bool aligned = (reinterpret_cast<uintptr_t>(img) % 16 == 0) &&
	                     (OP != OP_EM || reinterpret_cast<uintptr_t>(out) % 16 == 0) &&
	                     (h->P.g.nvox % 4 == 0);
	auto go = [&](auto tplc)
	{
		constexpr int TPL = decltype(tplc)::value;
		const uint64_t threads = R.count * TPL;
		const unsigned grid = static_cast<unsigned>(std::max<uint64_t>(1, (threads + B - 1) / B));
		if constexpr (TPL == 1 || K == K_SIDDON_MR)
		{
			// Bit 0: float4 gathers (forward); bit 1: float4 reductions summed
			// in registers, bit 2: staged in shared memory, bit 3: float2
			// pair reductions (back projection; bit 2 wins over bit 1, both
			// over bit 3).  Each op instantiates only the modes it uses;
			// multi-ray walks use the register float4 or pair reductions.
			constexpr int kUse = K == K_SIDDON_MR ? (OP == OP_FWD ? 0 : 10)
			                                      : (OP == OP_FWD ? 1 : (OP == OP_BWD ? 14 : 15));
			int vg = aligned ? (h->launch.vector_groups & kUse) : 0;
			if (vg & 4)
				vg &= ~2;
			if (vg & 6)
				vg &= ~8;
			if (vg != 0)
			{
				auto vlaunch = [&](auto vc)
				{
					constexpr int V = decltype(vc)::value;
					if constexpr ((V & kUse) == V)
						k_events<OP, K, T, C, false, B, TPL, V, TILE><<<grid, B, 0, st>>>(
						    h->P, E, R, in, out, gs, thr, h->d_err, F);
				};
				switch (vg)
				{
				case 1: vlaunch(std::integral_constant<int, 1>{}); break;
				case 2: vlaunch(std::integral_constant<int, 2>{}); break;
				case 3: vlaunch(std::integral_constant<int, 3>{}); break;
				case 4: vlaunch(std::integral_constant<int, 4>{}); break;
				case 5: vlaunch(std::integral_constant<int, 5>{}); break;
				case 8: vlaunch(std::integral_constant<int, 8>{}); break;
				default: vlaunch(std::integral_constant<int, 9>{}); break;
				}
				return;
			}
		}
		k_events<OP, K, T, C, false, B, TPL, 0, TILE><<<grid, B, 0, st>>>(h->P, E, R, in, out, gs,
		                                                        thr, h->d_err, F);
	};
	int tpl = h->launch.threads_per_lor;
	if constexpr (K == K_SIDDON_MR)
	{
		// One lane per ray reads its offsets from the table only: without a
		// table that covers the launch's items, one thread walks the rays.
		if (!(h->P.mrTable != nullptr && R.count <= h->P.mrCount))
			tpl = 1;
		if (tpl == 8)
			go(std::integral_constant<int, 8>{});
		else if (tpl == 4)
			go(std::integral_constant<int, 4>{});
		else if (tpl == 2)
			go(std::integral_constant<int, 2>{});
		else
			go(std::integral_constant<int, 1>{});
	}
	else if constexpr (C && !TILE)
	{
		if (tpl == 4)
			go(std::integral_constant<int, 4>{});
		else if (tpl == 2)
			go(std::integral_constant<int, 2>{});
		else
			go(std::integral_constant<int, 1>{});
	}
	else
	{
		// Tiled images: one thread per LOR.
		go(std::integral_constant<int, 1>{});
	}
}

// Lanes of the one-lane-per-ray multi-ray walk: the number of rays rounded
// up to a power of two; 0 above 8 rays (one thread then walks them all).
inline int rayLanes(int numRays)
{
	int l = 1;
	while (l < numRays)
		l <<= 1;
	return l <= 8 ? l : 0;
}

// layout: the images' layout (YRTB_LAYOUT_*), -1 for the projector's.
template <int OP>
yrtb_status dispatchEvents(yrtb_projector* h, const yrtb_events* ev,
                           yrtb_range range, const float* in, float* out,
                           float gs, float thr, yrtb_stream stream,
                           float* model = nullptr, int layout = -1)
{
	yrtb_status s = checkEvents(h, ev, range, true);
	if (s != YRTB_OK)
		return s;
	const bool tiled = OP != OP_COUNT && (layout < 0 ? h->layout : layout) == YRTB_LAYOUT_TILE_4X2;
	if (tiled && (h->kind != K_SIDDON || h->det))
		return fail(YRTB_ERR_ARGUMENT, "tiled images need a single-ray Siddon projector "
		                               "without deterministic back projection");
	if (range.count == 0)
		return YRTB_OK;
	YRTB_CUDA(cudaSetDevice(h->device));
	Events E = toDev(ev);
	E.model = model;
	const Range R{range.start, range.stride, range.count};
	cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
	constexpr bool kScatter = OP == OP_BWD || OP == OP_EM;
	Fixed F{};
	if (kScatter && h->det)
		if ((s = fixedBegin(h, R.count, st, F)) != YRTB_OK)
			return s;
	const unsigned grid = gridAll(R.count);
	withConfig(h, [&](auto kind, auto tof, auto comp)
	{
		constexpr int K = decltype(kind)::value;
		constexpr bool T = decltype(tof)::value;
		constexpr bool C = decltype(comp)::value;
		if constexpr (K == K_SIDDON && OP != OP_COUNT)
		{
			if (!(kScatter && h->det))
			{
				if (tiled)
				{
					if (h->launch.block == 128)
						launchTuned<OP, K, T, C, 128, true>(h, E, R, in, out, gs, thr, st, F);
					else
						launchTuned<OP, K, T, C, 256, true>(h, E, R, in, out, gs, thr, st, F);
				}
				else if (h->launch.block == 128)
					launchTuned<OP, K, T, C, 128>(h, E, R, in, out, gs, thr, st, F);
				else
					launchTuned<OP, K, T, C, 256>(h, E, R, in, out, gs, thr, st, F);
				return;
			}
		}
		if constexpr (K == K_SIDDON_MR && OP != OP_COUNT)
		{
			if (!(kScatter && h->det))
			{
				launchTuned<OP, K, T, C, kBlock>(h, E, R, in, out, gs, thr, st, F);
				return;
			}
		}
		if constexpr (kScatter)
		{
			if (h->det)
			{
				k_events_bound<OP == OP_EM, K, T, C><<<grid, kBlock, 0, st>>>(
				    h->P, E, R, in, gs, thr, h->d_fixMax);
				k_events<OP, K, T, C, true><<<grid, kBlock, 0, st>>>(
				    h->P, E, R, in, out, gs, thr, h->d_err, F);
				return;
			}
		}
		k_events<OP, K, T, C><<<grid, kBlock, 0, st>>>(h->P, E, R, in, out, gs,
		                                               thr, h->d_err, F);
	});
	if (kScatter && h->det)
		fixedEnd(h, F, out, st);
	YRTB_LAUNCHED();
	return YRTB_OK;
}

// Threads per bin of the compensated DD + PSF histogram EM pass (measured
// on a 12-subset OSEM iteration of a 1.8M-bin histogram: 1 thread 84.6 ms,
// 2: 80.0, 4: 76.8, 8: 78.5).
constexpr int kHistoDDThreads = 4;

// Bins of one subset that the histogram EM pass does work for: a valid
// detector pair and a non-zero measurement (NaN included), exactly the bins
// k_histo<EM> does not skip.
struct NonzeroBin
{
	H3Dev H;
	const float* meas;
	uint64_t nps, numSubsets, subset;
	__device__ bool operator()(uint64_t k) const
	{
		const uint64_t bin = h3SubsetBin(H, k, nps, numSubsets, subset);
		uint32_t d1, d2;
		h3Pair(H, bin, d1, d2);
		if (d1 == 0 && d2 == 0)
			return false;
		return !(__ldg(meas + bin) == 0.f);
	}
};

template <bool EM>
yrtb_status dispatchHisto(yrtb_projector* h, int numSubsets, int subset,
                          const float* img, float* out, const float* meas,
                          const float* sensH, const float* acfH,
                          const float* addH, const float* mu,
                          const yrtb_image_params* muParams, float gs,
                          float thr, yrtb_stream stream,
                          const uint64_t* list = nullptr, uint64_t listCount = 0,
                          const float* crystalEff = nullptr)
{
	if (!h || !out || numSubsets <= 0 || subset < 0 || subset >= numSubsets)
		return fail(YRTB_ERR_ARGUMENT, "invalid histogram subset or buffers");
	if (EM && (!img || !meas))
		return fail(YRTB_ERR_ARGUMENT, "histogram EM needs image and measurements");
	if (mu && !validImage(muParams))
		return fail(YRTB_ERR_ARGUMENT, "attenuation image needs valid parameters");
	if (h->ip.nt != 1)
		return fail(YRTB_ERR_ARGUMENT, "histogram-mode projection is single-frame");
	YRTB_CUDA(cudaSetDevice(h->device));
	uint64_t nps = 0;
	const uint64_t subsetCount = h3SubsetSize(*h->h3, numSubsets, subset, nps);
	// Threads: one per listed bin, or one per bin of the subset.  The
	// fixed-point scale of deterministic mode is set by the subset size in
	// both forms, so that they give the same image.
	const uint64_t count = list ? listCount : subsetCount;
	const Geom mg = mu ? makeGeom(*muParams) : Geom{};
	cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
	const unsigned grid = gridAll(count);
	Fixed F{};
	if (h->det)
	{
		const yrtb_status s = fixedBegin(h, subsetCount, st, F);
		if (s != YRTB_OK)
			return s;
	}
	auto launch = [&](auto kind, auto comp)
	{
		constexpr int K = decltype(kind)::value;
		constexpr bool C = decltype(comp)::value;
		if (h->det)
		{
			k_histo<K, EM, H_BOUND, C><<<grid, kBlock, 0, st>>>(
			    h->P, h->h3d, count, nps, numSubsets, subset, img, out, meas, sensH,
			    acfH, addH, mg, mu, gs, thr, F, h->d_fixMax, list, crystalEff);
			k_histo<K, EM, H_FIX, C><<<grid, kBlock, 0, st>>>(
			    h->P, h->h3d, count, nps, numSubsets, subset, img, out, meas, sensH,
			    acfH, addH, mg, mu, gs, thr, F, nullptr, list, crystalEff);
		}
		else if constexpr (EM && K == K_DD_PSF && C)
		{
			// Compensated DD + PSF EM: kHistoDDThreads threads per bin, each
			// on an even share of the bin's rows.
			constexpr int T = kHistoDDThreads;
			k_histo<K, EM, H_PLAIN, C, T><<<gridAll(count * T), kBlock, 0, st>>>(
			    h->P, h->h3d, count, nps, numSubsets, subset, img, out, meas, sensH,
			    acfH, addH, mg, mu, gs, thr, F, nullptr, list, crystalEff);
		}
		else
		{
			k_histo<K, EM, H_PLAIN, C><<<grid, kBlock, 0, st>>>(
			    h->P, h->h3d, count, nps, numSubsets, subset, img, out, meas, sensH,
			    acfH, addH, mg, mu, gs, thr, F, nullptr, list, crystalEff);
		}
	};
	// Histogram mode honours the precision for single-ray Siddon and DD + PSF.
	switch (h->kind)
	{
	case K_SIDDON:
		if (h->comp)
			launch(std::integral_constant<int, K_SIDDON>{}, std::true_type{});
		else
			launch(std::integral_constant<int, K_SIDDON>{}, std::false_type{});
		break;
	case K_SIDDON_MR: launch(std::integral_constant<int, K_SIDDON_MR>{}, std::false_type{}); break;
	case K_DD: launch(std::integral_constant<int, K_DD>{}, std::false_type{}); break;
	default:
		if (h->comp)
			launch(std::integral_constant<int, K_DD_PSF>{}, std::true_type{});
		else
			launch(std::integral_constant<int, K_DD_PSF>{}, std::false_type{});
		break;
	}
	if (h->det)
		fixedEnd(h, F, out, st);
	YRTB_LAUNCHED();
	return YRTB_OK;
}

// Subset-major permutation of the events (see yrtb_events_subset_order)
// with the ordering parameters of cfg.
yrtb_status orderEvents(yrtb_projector* h, const yrtb_events* ev, uint64_t S,
                        const yrtb_launch_config& cfg, uint64_t* d_perm,
                        cudaStream_t st, uint64_t first = 0)
{
	const uint64_t n = ev->count;
	if (n == 0)
		return YRTB_OK;
	YRTB_CUDA(cudaSetDevice(h->device));
	unsigned long long *keys = nullptr, *keys2 = nullptr, *vals = nullptr;
	uint32_t *v32 = nullptr, *v32b = nullptr;
	void* temp = nullptr;
	size_t tempBytes = 0;
	// Event indices as 32-bit values when they fit (a quarter less traffic
	// per radix pass), widened into d_perm after the sort.
	const bool small = n <= 0xffffffffull;
	auto release = [&]
	{
		cudaFreeAsync(keys, st);
		cudaFreeAsync(keys2, st);
		cudaFreeAsync(vals, st);
		cudaFreeAsync(v32, st);
		cudaFreeAsync(v32b, st);
		cudaFreeAsync(temp, st);
	};
	cudaError_t ce = poolAlloc(&keys, n * 8, st);
	if (ce == cudaSuccess)
		ce = poolAlloc(&keys2, n * 8, st);
	if (ce == cudaSuccess && small)
		ce = poolAlloc(&v32, n * 4, st);
	if (ce == cudaSuccess && small)
		ce = poolAlloc(&v32b, n * 4, st);
	if (ce == cudaSuccess && !small)
		ce = poolAlloc(&vals, n * 8, st);
	if (ce != cudaSuccess)
	{
		release();
		return fail(YRTB_ERR_CUDA, cudaGetErrorString(ce));
	}
	// Estimated crossings of the single-ray Siddon walk (into keys2, which
	// the sort overwrites afterwards): O(1) per event instead of a walk.
	const uint32_t* counts = nullptr;
	if (h->kind == K_SIDDON && (!h->hasTof || ev->tof_ps))
	{
		uint32_t* c32 = reinterpret_cast<uint32_t*>(keys2);
		if (h->hasTof)
			k_count_estimate<true><<<gridFor(n, 16), kBlock, 0, st>>>(h->P, toDev(ev), n, c32);
		else
			k_count_estimate<false><<<gridFor(n, 16), kBlock, 0, st>>>(h->P, toDev(ev), n, c32);
		counts = c32;
	}
	// LOR keys wider than their field keep their high bits.
	const int lorBits = ev->frame ? 29 : 33;
	const uint64_t nd = h->h3d.numDets;
	const uint64_t maxKey = h->h3 ? h->h3->numZBin * h->h3->numPhi * h->h3->numR
	                              : nd * nd;
	int keyBits = 0;
	while (keyBits < 64 && (maxKey >> keyBits) != 0)
		keyBits++;
	const int lorShift = std::max(0, keyBits - lorBits);
	const float voxel = std::max(h->P.g.vx, std::max(h->P.g.vy, h->P.g.vz));
	const float cell = voxel * static_cast<float>(1 << cfg.tile_shift);
	k_order_keys<<<gridFor(n, 16), kBlock, 0, st>>>(
	    h->P, h->h3d, h->h3 != nullptr, toDev(ev), n, S, first % S, counts,
	    cfg.bucket_shift, lorShift, cfg.order, cell, keys, vals, v32);
	// Only the key bits in use are sorted: the subset field ends at bit
	// (frames ? 52 : 48) + bits(S - 1), 8 bits lower for the spatial orders.
	int sBits = 0;
	while (sBits < 16 && ((S - 1) >> sBits) != 0)
		sBits++;
	const int endBit = std::min(64, (ev->frame ? 52 : 48) - (cfg.order != YRTB_ORDER_LOR ? 8 : 0) +
	                                    sBits);
	auto* perm64 = reinterpret_cast<unsigned long long*>(d_perm);
	auto sortPairs = [&](void* t, size_t& bytes)
	{
		return small ? cub::DeviceRadixSort::SortPairs(t, bytes, keys, keys2, v32, v32b, n, 0,
		                                               endBit, st)
		             : cub::DeviceRadixSort::SortPairs(t, bytes, keys, keys2, vals, perm64, n,
		                                               0, endBit, st);
	};
	ce = sortPairs(nullptr, tempBytes);
	if (ce == cudaSuccess)
		ce = poolAlloc(&temp, tempBytes, st);
	if (ce == cudaSuccess)
		ce = sortPairs(temp, tempBytes);
	if (ce == cudaSuccess && small)
	{
		k_widen_u32<<<gridFor(n, 16), kBlock, 0, st>>>(v32b, n, perm64);
		ce = cudaGetLastError();
	}
	release();
	if (ce != cudaSuccess)
		return fail(YRTB_ERR_CUDA, cudaGetErrorString(ce));
	YRTB_LAUNCHED();
	return YRTB_OK;
}

yrtb_status scannerCheck(const yrtb_scanner* s)
{
	if (!s)
		return fail(YRTB_ERR_ARGUMENT, "null scanner");
	if (s->dets_per_ring == 0 || s->num_rings == 0 || s->num_doi == 0 ||
	    s->dets_per_block == 0 || s->dets_per_ring % s->dets_per_block != 0)
		return fail(YRTB_ERR_ARGUMENT, "invalid scanner detector counts");
	if (s->max_ring_diff >= s->num_rings)
		return fail(YRTB_ERR_ARGUMENT,
		            "Maximum Ring difference has to be lower than the number of rings");
	if (s->min_ang_diff == 0)
		return fail(YRTB_ERR_ARGUMENT, "Minimum angle difference has to be non-zero");
	const uint64_t nd = s->dets_per_ring * s->num_rings * s->num_doi;
	if (nd >= (uint64_t(1) << 32))
		return fail(YRTB_ERR_ARGUMENT, "too many detectors for 32-bit ids");
	return YRTB_OK;
}

}  // namespace

// ================================================================ C ABI ===
extern "C" {

const char* yrtb_last_error(void)
{
	return g_lastError.c_str();
}

int yrtb_version(void)
{
	return 1;
}

yrtb_status yrtb_scanner_regular_lut(const yrtb_scanner* s, float* out)
{
	yrtb_status st = scannerCheck(s);
	if (st != YRTB_OK)
		return st;
	if (!out)
		return fail(YRTB_ERR_ARGUMENT, "null output");
	// DetRegular::generateLUT (DetRegular.cpp:113-183), float arithmetic with
	// the reference's double constants.
	const double PI_ = 3.14159265358979;
	const double TWOPI_ = 6.28318530717959;
	const size_t numBlocks = s->dets_per_ring / s->dets_per_block;
	const float blockLength = s->crystal_size_trans * s->dets_per_block;
	for (size_t doi = 0; doi < s->num_doi; doi++)
	{
		const float blockDistance = s->scanner_radius + s->crystal_depth * doi;
		for (size_t ring = 0; ring < s->num_rings; ring++)
		{
			const float zGap = s->axial_fov / static_cast<float>(s->num_rings);
			const float zPos = -s->axial_fov / 2.0 + (ring + 0.5f) * zGap;
			for (size_t block = 0; block < numBlocks; block++)
			{
				const float angle = block * TWOPI_ / numBlocks;
				const float xb = (blockDistance + 0.5f * s->crystal_depth) * std::cos(angle);
				const float yb = (blockDistance + 0.5f * s->crystal_depth) * std::sin(angle);
				for (size_t det = 0; det < s->dets_per_block; det++)
				{
					float rel = 0.0f;
					if (s->dets_per_block != 1)
						rel = -0.5 + (det + 0.5) / static_cast<float>(s->dets_per_block);
					const float rx = rel * std::cos(angle + PI_ / 2.0);
					const float ry = rel * std::sin(angle + PI_ / 2.0);
					const size_t idx = det + block * s->dets_per_block +
					                   ring * s->dets_per_ring +
					                   doi * (s->num_rings * s->dets_per_ring);
					out[idx * 6 + 0] = xb + blockLength * rx;
					out[idx * 6 + 1] = yb + blockLength * ry;
					out[idx * 6 + 2] = zPos;
					out[idx * 6 + 3] = std::cos(angle);
					out[idx * 6 + 4] = std::sin(angle);
					out[idx * 6 + 5] = 0.0f;
				}
			}
		}
	}
	return YRTB_OK;
}

yrtb_status yrtb_histo3d_dims(const yrtb_scanner* s, uint64_t* dims)
{
	yrtb_status st = scannerCheck(s);
	if (st != YRTB_OK)
		return st;
	if (s->dets_per_ring % 2 != 0)
		return fail(YRTB_ERR_ARGUMENT,
		            "The number of detectors per ring has to be even");
	H3Host h(*s);
	dims[0] = h.numZBin;
	dims[1] = h.numPhi;
	dims[2] = h.numR;
	return YRTB_OK;
}

yrtb_status yrtb_projector_create(const yrtb_scanner* s, const float* lut,
                                  const yrtb_image_params* ip,
                                  const yrtb_projector_params* pp,
                                  yrtb_projector** out)
{
	if (!out)
		return fail(YRTB_ERR_ARGUMENT, "null output handle");
	*out = nullptr;
	yrtb_status st = scannerCheck(s);
	if (st != YRTB_OK)
		return st;
	if (!validImage(ip))
		return fail(YRTB_ERR_ARGUMENT, "invalid image parameters");
	if (!pp || (pp->projector != YRTB_SIDDON && pp->projector != YRTB_DD))
		return fail(YRTB_ERR_ARGUMENT, "unknown projector type");
	if (pp->num_rays < 1)
		return fail(YRTB_ERR_ARGUMENT, "num_rays must be >= 1");
	if (pp->psf_num_s > 0 && (!pp->psf_taps || pp->psf_size <= 0 ||
	                          pp->psf_size % 2 == 0 || pp->psf_k_spacing <= 0 ||
	                          pp->psf_s_step <= 0))
		return fail(YRTB_ERR_ARGUMENT, "Kernels must be of odd length (invalid PSF table)");
	if (pp->precision != YRTB_MIRROR && pp->precision != YRTB_COMPENSATED)
		return fail(YRTB_ERR_ARGUMENT, "unknown precision mode");

	auto h = std::make_unique<yrtb_projector>();
	h->sc = *s;
	h->ip = *ip;
	h->pp = *pp;
	h->pp.psf_taps = nullptr;
	cudaGetDevice(&h->device);
	const uint64_t nd = s->dets_per_ring * s->num_rings * s->num_doi;
	std::vector<float> hl(nd * 6);
	if (lut)
		std::memcpy(hl.data(), lut, nd * 6 * sizeof(float));
	else
		yrtb_scanner_regular_lut(s, hl.data());
	std::vector<float4> pos(nd), ori(nd);
	for (uint64_t d = 0; d < nd; d++)
	{
		pos[d] = make_float4(hl[d * 6 + 0], hl[d * 6 + 1], hl[d * 6 + 2], 0.f);
		ori[d] = make_float4(hl[d * 6 + 3], hl[d * 6 + 4], hl[d * 6 + 5], 0.f);
	}
	YRTB_CUDA(cudaMalloc(&h->d_pos, nd * sizeof(float4)));
	YRTB_CUDA(cudaMalloc(&h->d_ori, nd * sizeof(float4)));
	YRTB_CUDA(cudaMemcpy(h->d_pos, pos.data(), nd * sizeof(float4), cudaMemcpyHostToDevice));
	YRTB_CUDA(cudaMemcpy(h->d_ori, ori.data(), nd * sizeof(float4), cudaMemcpyHostToDevice));
	YRTB_CUDA(cudaMalloc(&h->d_err, sizeof(unsigned long long)));
	YRTB_CUDA(cudaMemset(h->d_err, 0, sizeof(unsigned long long)));

	KParams& P = h->P;
	P.g = makeGeom(*ip);
	P.scan.pos = h->d_pos;
	P.scan.ori = h->d_ori;
	P.scan.numDets = static_cast<uint32_t>(nd);
	P.scan.crystalZ = s->crystal_size_z;
	P.scan.crystalTrans = s->crystal_size_trans;
	P.numRays = pp->num_rays;
	P.mrTable = nullptr;
	P.mrCount = 0;
	h->hasTof = pp->tof_fwhm_ps > 0.f;
	if (h->hasTof)
	{
		// TimeOfFlightHelper constructor (TimeOfFlight.hpp:20-34).
		const double w_mm = pp->tof_fwhm_ps * kSpeedOfLightMmPs * 0.5;
		P.tof.sigma = static_cast<float>(w_mm / (2 * sqrtf(2 * logf(2))));
		P.tof.trunc = (pp->tof_n_std <= 0) ? -1.f : pp->tof_n_std * P.tof.sigma;
		P.tof.norm = static_cast<float>(1 / (std::sqrt(2 * 3.14159265358979) * P.tof.sigma));
	}
	h->comp = pp->precision == YRTB_COMPENSATED;
	h->det = pp->deterministic != 0;
	if (h->det)
	{
		const uint64_t J = static_cast<uint64_t>(P.g.nvox) * ip->nt;
		YRTB_CUDA(cudaMalloc(&h->d_fix, J * sizeof(unsigned long long)));
		YRTB_CUDA(cudaMalloc(&h->d_fixMax, sizeof(unsigned)));
	}
	if (pp->projector == YRTB_SIDDON)
		h->kind = pp->num_rays > 1 ? K_SIDDON_MR : K_SIDDON;
	else
		h->kind = pp->psf_num_s > 0 ? K_DD_PSF : K_DD;
	// Multi-ray Siddon walks one ray per lane by default (up to 8 rays) and
	// sends its back projection as pairs of voxels (C2, 4 rays: 97.3 ms per
	// OSEM iteration against 101.2 ms with float4 groups).
	if (h->kind == K_SIDDON_MR && rayLanes(pp->num_rays) > 0)
	{
		h->launch.threads_per_lor = rayLanes(pp->num_rays);
		h->launch.vector_groups = 8;
	}
	if (pp->psf_num_s > 0)
	{
		const size_t n = static_cast<size_t>(pp->psf_num_s) * pp->psf_size;
		std::vector<float> flipped(n);
		for (int i = 0; i < pp->psf_num_s; i++)
			for (int j = 0; j < pp->psf_size; j++)
				flipped[i * pp->psf_size + pp->psf_size - 1 - j] =
				    pp->psf_taps[i * pp->psf_size + j];
		YRTB_CUDA(cudaMalloc(&h->d_taps, n * sizeof(float)));
		YRTB_CUDA(cudaMalloc(&h->d_flipped, n * sizeof(float)));
		YRTB_CUDA(cudaMemcpy(h->d_taps, pp->psf_taps, n * sizeof(float), cudaMemcpyHostToDevice));
		YRTB_CUDA(cudaMemcpy(h->d_flipped, flipped.data(), n * sizeof(float), cudaMemcpyHostToDevice));
		// Prefix sums of the trapezoid bins per kernel row (FP64, stored FP32).
		const int K = pp->psf_size, W = K + 3;
		auto prefixOf = [&](const std::vector<float>& t, std::vector<float>& out)
		{
			out.assign(static_cast<size_t>(pp->psf_num_s) * W, 0.f);
			for (int i = 0; i < pp->psf_num_s; i++)
			{
				auto v = [&](int k) { return (k < 0 || k >= K) ? 0.0 : double(t[size_t(i) * K + k]); };
				double acc = 0.0;
				out[size_t(i) * W + 0] = 0.f;
				for (int m = 1; m < W; m++)
				{
					const int xi = m - 2;
					if (xi >= -1)
						acc += double(pp->psf_k_spacing) * 0.5 * (v(xi) + v(xi + 1));
					out[size_t(i) * W + m] = static_cast<float>(acc);
				}
			}
		};
		std::vector<float> taps(pp->psf_taps, pp->psf_taps + n), pre, preF;
		prefixOf(taps, pre);
		prefixOf(flipped, preF);
		YRTB_CUDA(cudaMalloc(&h->d_prefix, pre.size() * sizeof(float)));
		YRTB_CUDA(cudaMalloc(&h->d_prefixFlipped, preF.size() * sizeof(float)));
		YRTB_CUDA(cudaMemcpy(h->d_prefix, pre.data(), pre.size() * sizeof(float), cudaMemcpyHostToDevice));
		YRTB_CUDA(cudaMemcpy(h->d_prefixFlipped, preF.data(), preF.size() * sizeof(float), cudaMemcpyHostToDevice));
		P.psf = Psf{h->d_taps, h->d_flipped, pp->psf_num_s, pp->psf_size,
		            pp->psf_s_step, pp->psf_k_spacing, h->d_prefix, h->d_prefixFlipped};
	}
	h->h3d.numDets = static_cast<uint32_t>(nd);
	if (s->dets_per_ring % 2 == 0)
	{
		h->h3 = std::make_unique<H3Host>(*s);
		const H3Host& H = *h->h3;
		YRTB_CUDA(cudaMalloc(&h->d_ring, H.ringMap.size() * sizeof(int32_t)));
		YRTB_CUDA(cudaMalloc(&h->d_z, H.zPairs.size() * sizeof(int2)));
		YRTB_CUDA(cudaMemcpy(h->d_ring, H.ringMap.data(), H.ringMap.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
		YRTB_CUDA(cudaMemcpy(h->d_z, H.zPairs.data(), H.zPairs.size() * sizeof(int2), cudaMemcpyHostToDevice));
		h->h3d = H3Dev{static_cast<uint32_t>(nd), h->d_ring, h->d_z, static_cast<uint32_t>(H.dpr),
		               static_cast<uint32_t>(H.rings), static_cast<uint32_t>(H.ndoi),
		               static_cast<uint32_t>(H.numDOIPoss), static_cast<uint32_t>(H.rCut),
		               static_cast<uint32_t>(H.mrd), H.numR, H.numPhi, H.numZBin,
		               H.numZBinDiff};
	}
	*out = h.release();
	return YRTB_OK;
}

void yrtb_projector_destroy(yrtb_projector* h)
{
	delete h;
}

yrtb_status yrtb_release_cached_memory(void)
{
	std::lock_guard<std::mutex> guard(g_poolLock);
	for (int d = 0; d < kMaxPoolDevices; d++)
		if (g_pools[d] != nullptr)
		{
			int cur = 0;
			YRTB_CUDA(cudaGetDevice(&cur));
			YRTB_CUDA(cudaSetDevice(d));
			YRTB_CUDA(cudaDeviceSynchronize());
			YRTB_CUDA(cudaMemPoolTrimTo(g_pools[d], 0));
			YRTB_CUDA(cudaSetDevice(cur));
		}
	return YRTB_OK;
}

yrtb_status yrtb_projector_set_launch(yrtb_projector* h,
                                      const yrtb_launch_config* c)
{
	if (!h || !c)
		return fail(YRTB_ERR_ARGUMENT, "null argument");
	if (c->block != 128 && c->block != 256)
		return fail(YRTB_ERR_ARGUMENT, "block must be 128 or 256");
	if (h->kind == K_SIDDON_MR)
	{
		if (c->threads_per_lor != 1 && c->threads_per_lor != rayLanes(h->P.numRays))
			return fail(YRTB_ERR_ARGUMENT,
			            "threads_per_lor of a multi-ray Siddon projector must be 1 or "
			            "the number of rays rounded up to a power of two (at most 8)");
	}
	else
	{
		if (c->threads_per_lor != 1 && c->threads_per_lor != 2 && c->threads_per_lor != 4)
			return fail(YRTB_ERR_ARGUMENT, "threads_per_lor must be 1, 2 or 4");
		if (c->threads_per_lor > 1 && !(h->kind == K_SIDDON && h->comp))
			return fail(YRTB_ERR_ARGUMENT,
			            "threads_per_lor > 1 needs a single-ray Siddon projector in "
			            "YRTB_COMPENSATED precision, or a multi-ray one");
	}
	if (c->bucket_shift < 0 || c->bucket_shift > 7)
		return fail(YRTB_ERR_ARGUMENT, "bucket_shift must be in 0..7");
	if (c->order != YRTB_ORDER_LOR && c->order != YRTB_ORDER_SPATIAL &&
	    c->order != YRTB_ORDER_SPATIAL_FINE)
		return fail(YRTB_ERR_ARGUMENT,
		            "order must be YRTB_ORDER_LOR, YRTB_ORDER_SPATIAL or YRTB_ORDER_SPATIAL_FINE");
	if (c->tile_shift < 0 || c->tile_shift > 4)
		return fail(YRTB_ERR_ARGUMENT, "tile_shift must be in 0..4");
	if (c->vector_groups < 0 || c->vector_groups > 15)
		return fail(YRTB_ERR_ARGUMENT, "vector_groups must be in 0..15");
	h->launch = *c;
	return YRTB_OK;
}

yrtb_status yrtb_projector_get_launch(const yrtb_projector* h,
                                      yrtb_launch_config* c)
{
	if (!h || !c)
		return fail(YRTB_ERR_ARGUMENT, "null argument");
	*c = h->launch;
	return YRTB_OK;
}

yrtb_status yrtb_projector_set_image_layout(yrtb_projector* h, int layout)
{
	if (!h)
		return fail(YRTB_ERR_ARGUMENT, "null projector");
	if (layout != YRTB_LAYOUT_ROW_MAJOR && layout != YRTB_LAYOUT_TILE_4X2)
		return fail(YRTB_ERR_ARGUMENT, "unknown image layout");
	if (layout == YRTB_LAYOUT_TILE_4X2)
	{
		if (h->kind != K_SIDDON || h->det)
			return fail(YRTB_ERR_ARGUMENT, "tiled images need a single-ray Siddon "
			                               "projector without deterministic back projection");
		if (h->ip.nx % 4 != 0 || h->ip.ny % 2 != 0)
			return fail(YRTB_ERR_ARGUMENT, "tiled images need nx % 4 == 0 and ny % 2 == 0");
	}
	h->layout = layout;
	return YRTB_OK;
}

yrtb_status yrtb_projector_get_image_layout(const yrtb_projector* h, int* layout)
{
	if (!h || !layout)
		return fail(YRTB_ERR_ARGUMENT, "null argument");
	*layout = h->layout;
	return YRTB_OK;
}

yrtb_status yrtb_image_convert_layout(const float* d_src, float* d_dst,
                                      const yrtb_image_params* ip, int to_layout,
                                      yrtb_stream stream)
{
	if (!d_src || !d_dst || d_src == d_dst || !validImage(ip))
		return fail(YRTB_ERR_ARGUMENT, "invalid layout conversion arguments");
	if (to_layout != YRTB_LAYOUT_ROW_MAJOR && to_layout != YRTB_LAYOUT_TILE_4X2)
		return fail(YRTB_ERR_ARGUMENT, "unknown image layout");
	if (ip->nx % 4 != 0 || ip->ny % 2 != 0)
		return fail(YRTB_ERR_ARGUMENT, "tiled images need nx % 4 == 0 and ny % 2 == 0");
	const uint64_t total = static_cast<uint64_t>(ip->nx) * ip->ny * ip->nz * ip->nt;
	cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
	const unsigned grid = static_cast<unsigned>((total + kBlock - 1) / kBlock);
	if (to_layout == YRTB_LAYOUT_TILE_4X2)
		k_convert_layout<true><<<grid, kBlock, 0, st>>>(d_src, d_dst, ip->nx, ip->ny, ip->nz, total);
	else
		k_convert_layout<false><<<grid, kBlock, 0, st>>>(d_src, d_dst, ip->nx, ip->ny, ip->nz, total);
	YRTB_LAUNCHED();
	return YRTB_OK;
}

yrtb_status yrtb_multiray_offsets(yrtb_projector* h, uint64_t count,
                                  float* d_out, yrtb_stream stream)
{
	if (!h || !d_out)
		return fail(YRTB_ERR_ARGUMENT, "null argument");
	if (h->P.numRays < 2 || count == 0)
		return YRTB_OK;
	YRTB_CUDA(cudaSetDevice(h->device));
	k_multiray_offsets<<<gridAll(count), kBlock, 0,
	                     reinterpret_cast<cudaStream_t>(stream)>>>(
	    count, h->P.numRays, d_out);
	YRTB_LAUNCHED();
	return YRTB_OK;
}

yrtb_status yrtb_multiray_table(yrtb_projector* h, uint64_t count,
                                yrtb_stream stream)
{
	if (!h)
		return fail(YRTB_ERR_ARGUMENT, "null projector");
	if (h->P.numRays < 2 || count <= h->mrCapacity)
		return YRTB_OK;
	YRTB_CUDA(cudaSetDevice(h->device));
	cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
	// Launches already queued may still read the old table.
	YRTB_CUDA(cudaDeviceSynchronize());
	h->P.mrTable = nullptr;
	h->P.mrCount = 0;
	YRTB_CUDA(cudaFree(h->d_mrTable));
	h->d_mrTable = nullptr;
	h->mrCapacity = 0;
	const uint64_t per = 4 * static_cast<uint64_t>(h->P.numRays - 1);
	YRTB_CUDA(cudaMalloc(&h->d_mrTable, count * per * sizeof(float)));
	k_multiray_offsets<<<gridAll(count), kBlock, 0, st>>>(count, h->P.numRays,
	                                                       h->d_mrTable);
	YRTB_LAUNCHED();
	h->mrCapacity = count;
	h->P.mrTable = h->d_mrTable;
	h->P.mrCount = count;
	return YRTB_OK;
}

yrtb_status yrtb_events_subset_order_from(yrtb_projector* h, const yrtb_events* ev,
                                          int num_subsets,
                                          uint64_t first_global_index,
                                          uint64_t* d_perm, uint64_t* subset_offsets,
                                          yrtb_stream stream)
{
	if (!h || !ev || (!d_perm && ev->count > 0) || !subset_offsets || num_subsets <= 0 ||
	    num_subsets > (ev->frame ? 4095 : 65535))
		return fail(YRTB_ERR_ARGUMENT, "invalid subset-order arguments");
	const uint64_t n = ev->count;
	const uint64_t S = static_cast<uint64_t>(num_subsets);
	const uint64_t r = first_global_index % S;
	// Subset s holds the local events e with (r + e) mod S == s: the first
	// is e = (s - r) mod S, then every S-th.
	subset_offsets[0] = 0;
	for (uint64_t s = 0; s < S; s++)
	{
		const uint64_t k = (s + S - r) % S;
		subset_offsets[s + 1] = subset_offsets[s] + (n > k ? (n - k + S - 1) / S : 0);
	}
	return orderEvents(h, ev, S, h->launch, d_perm,
	                   reinterpret_cast<cudaStream_t>(stream), first_global_index);
}

yrtb_status yrtb_events_subset_order(yrtb_projector* h, const yrtb_events* ev,
                                     int num_subsets, uint64_t* d_perm,
                                     uint64_t* subset_offsets,
                                     yrtb_stream stream)
{
	return yrtb_events_subset_order_from(h, ev, num_subsets, 0, d_perm,
	                                     subset_offsets, stream);
}

}  // extern "C"

namespace
{
// out->X[i] = in->X[d_perm[i]].  packable: d_perm is a permutation of
// 0..count-1, so the source arrays may be interleaved into 16-byte records
// first (one random sector per event); otherwise (a perm that reaches
// beyond count, e.g. every S-th event of a longer array) the arrays are read
// directly.
yrtb_status gatherEvents(const yrtb_events* in, const uint64_t* d_perm,
                         const yrtb_events* out, yrtb_stream stream, bool packable)
{
	if (!in || !out)
		return fail(YRTB_ERR_ARGUMENT, "invalid gather arguments");
	const uint64_t n = in->count;
	if (out->count != n)
		return fail(YRTB_ERR_ARGUMENT, "gather needs equal event counts");
	if (n == 0)
		return YRTB_OK;
	if (!d_perm)
		return fail(YRTB_ERR_ARGUMENT, "invalid gather arguments");
	cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
	const unsigned long long* perm = reinterpret_cast<const unsigned long long*>(d_perm);
	auto g32 = [&](const void* a, const void* b, int w) -> yrtb_status
	{
		if (a == nullptr)
			return YRTB_OK;
		if (b == nullptr)
			return fail(YRTB_ERR_ARGUMENT, "gather output array missing");
		k_gather<uint32_t><<<gridFor(n * w, 16), kBlock, 0, st>>>(
		    static_cast<const uint32_t*>(a), perm, n, w,
		    const_cast<uint32_t*>(static_cast<const uint32_t*>(b)));
		return YRTB_OK;
	};
	GatherSet G{};
	auto add = [&](const void* a, const void* b) -> yrtb_status
	{
		if (a == nullptr)
			return YRTB_OK;
		if (b == nullptr)
			return fail(YRTB_ERR_ARGUMENT, "gather output array missing");
		G.src[G.count] = static_cast<const uint32_t*>(a);
		G.dst[G.count] = const_cast<uint32_t*>(static_cast<const uint32_t*>(b));
		G.count++;
		return YRTB_OK;
	};
	yrtb_status r;
	if ((r = add(in->d1, out->d1)) || (r = add(in->d2, out->d2)) ||
	    (r = add(in->tof_ps, out->tof_ps)) || (r = add(in->frame, out->frame)) ||
	    (r = add(in->motion_frame, out->motion_frame)) ||
	    (r = add(in->measurement, out->measurement)) ||
	    (r = add(in->sens, out->sens)) || (r = add(in->att, out->att)) ||
	    (r = add(in->additive, out->additive)) || (r = g32(in->lor, out->lor, 6)) ||
	    (r = g32(in->orient, out->orient, 6)))
		return r;
	if (G.count == 1)
	{
		k_gather_set<<<gridFor(n, 16), kBlock, 0, st>>>(G, perm, n);
	}
	else if (G.count > 1 && !packable)
	{
		k_gather_set<<<gridFor(n, 16), kBlock, 0, st>>>(G, perm, n);
	}
	else if (G.count > 1)
	{
		// Groups of up to four arrays: pack, then one 16-byte random read per
		// event (four 4-byte random reads cost four sectors).
		uint4* packed = nullptr;
		const cudaError_t ce = poolAlloc(&packed, n * sizeof(uint4), st);
		if (ce != cudaSuccess)
		{
			(void)cudaGetLastError();  // no room for the records: read directly
			k_gather_set<<<gridFor(n, 16), kBlock, 0, st>>>(G, perm, n);
		}
		else
		{
			for (int first = 0; first < G.count; first += 4)
			{
				const int cnt = std::min(4, G.count - first);
				k_pack4<<<gridFor(n, 16), kBlock, 0, st>>>(G, first, cnt, n, packed);
				k_unpack4_gather<<<gridFor(n, 16), kBlock, 0, st>>>(G, first, cnt, n,
				                                                      packed, perm);
			}
			cudaFreeAsync(packed, st);
		}
	}
	YRTB_LAUNCHED();
	return YRTB_OK;
}

}  // namespace

extern "C" {

// Byte offsets of the properties of one row (-1: absent), as yrtb_row_layout.
struct RowLayout
{
	uint32_t bytes;
	int lor, orient, tof, frame, meas, sens, att, rnd, sct;
};

// One event per thread: its row's properties into the structure of arrays.
// Rows are packed 4-byte words, so every field is read as 32-bit words.
__global__ void __launch_bounds__(kBlock)
    k_events_from_rows(const uint8_t* __restrict__ rows, uint64_t n, RowLayout L,
                       float* lor, float* orient, float* tof, int32_t* frame,
                       float* meas, float* sens, float* att, float* add)
{
	const uint64_t e = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	if (e >= n)
		return;
	const uint8_t* r = rows + e * L.bytes;
	auto f = [&](int off) { return __ldg(reinterpret_cast<const float*>(r + off)); };
	for (int k = 0; k < 6; k++)
		lor[e * 6 + k] = f(L.lor + 4 * k);
	if (orient)
		for (int k = 0; k < 6; k++)
			orient[e * 6 + k] = f(L.orient + 4 * k);
	if (tof)
		tof[e] = f(L.tof);
	if (frame)
		frame[e] = __ldg(reinterpret_cast<const int32_t*>(r + L.frame));
	if (meas)
		meas[e] = f(L.meas);
	if (sens)
		sens[e] = f(L.sens);
	if (att)
		att[e] = f(L.att);
	if (add)
	{
		// randoms + scatter: the reference adds them to the model one after
		// the other (OSEM_GPU.cu:1283-1295); one sum here, at most one
		// rounding apart.
		float a = 0.f;
		if (L.rnd >= 0)
			a = f(L.rnd);
		if (L.sct >= 0)
			a = (L.rnd >= 0) ? a + f(L.sct) : f(L.sct);
		add[e] = a;
	}
}

yrtb_status yrtb_events_from_rows(const void* d_rows, uint64_t count,
                                  const yrtb_row_layout* layout,
                                  const yrtb_events* out, yrtb_stream stream)
{
	if (!layout || !out)
		return fail(YRTB_ERR_ARGUMENT, "null row layout or events");
	if (count == 0)
		return YRTB_OK;
	if (!d_rows || !out->lor)
		return fail(YRTB_ERR_ARGUMENT, "rows and an LOR output are required");
	const yrtb_row_layout& l = *layout;
	if (l.row_bytes == 0 || l.row_bytes % 4 != 0 ||
	    reinterpret_cast<uintptr_t>(d_rows) % 4 != 0)
		return fail(YRTB_ERR_ARGUMENT, "rows must be 4-byte aligned and a "
		                               "multiple of 4 bytes long");
	auto bad = [&](int32_t off, uint32_t words) {
		return off < 0 || off % 4 != 0 ||
		       static_cast<uint64_t>(off) + 4u * words > l.row_bytes;
	};
	if (bad(l.lor, 6))
		return fail(YRTB_ERR_ARGUMENT, "rows hold no LOR");
	struct Want
	{
		const void* out;
		int32_t off;
		uint32_t words;
		const char* name;
	} want[] = {{out->orient, l.det_orient, 6, "DET_ORIENT"},
	            {out->tof_ps, l.tof, 1, "TOF"},
	            {out->frame, l.dynamic_frame, 1, "DYNAMIC_FRAME"},
	            {out->measurement, l.measurement, 1, "MEASUREMENT"},
	            {out->sens, l.sensitivity, 1, "SENSITIVITY"},
	            {out->att, l.attenuation, 1, "ATTENUATION"}};
	for (const Want& w : want)
		if (w.out && bad(w.off, w.words))
			return fail(YRTB_ERR_ARGUMENT,
			            std::string("rows hold no ") + w.name + " property");
	if (out->additive && bad(l.randoms, 1) && bad(l.scatter, 1))
		return fail(YRTB_ERR_ARGUMENT, "rows hold no randoms or scatter estimate");
	RowLayout L{l.row_bytes, l.lor, l.det_orient, l.tof, l.dynamic_frame,
	            l.measurement, l.sensitivity, l.attenuation,
	            bad(l.randoms, 1) ? -1 : l.randoms, bad(l.scatter, 1) ? -1 : l.scatter};
	k_events_from_rows<<<gridAll(count), kBlock, 0,
	                     reinterpret_cast<cudaStream_t>(stream)>>>(
	    static_cast<const uint8_t*>(d_rows), count, L, const_cast<float*>(out->lor),
	    const_cast<float*>(out->orient), const_cast<float*>(out->tof_ps),
	    const_cast<int32_t*>(out->frame), const_cast<float*>(out->measurement),
	    const_cast<float*>(out->sens), const_cast<float*>(out->att),
	    const_cast<float*>(out->additive));
	YRTB_LAUNCHED();
	return YRTB_OK;
}

yrtb_status yrtb_events_gather(const yrtb_events* in, const uint64_t* d_perm,
                               const yrtb_events* out, yrtb_stream stream)
{
	return gatherEvents(in, d_perm, out, stream, true);
}

yrtb_status yrtb_projector_take_event_errors(yrtb_projector* h, uint64_t* count)
{
	if (!h || !count)
		return fail(YRTB_ERR_ARGUMENT, "null argument");
	unsigned long long v = 0;
	YRTB_CUDA(cudaSetDevice(h->device));
	YRTB_CUDA(cudaMemcpy(&v, h->d_err, sizeof(v), cudaMemcpyDeviceToHost));
	YRTB_CUDA(cudaMemset(h->d_err, 0, sizeof(v)));
	*count = v;
	return YRTB_OK;
}

yrtb_status yrtb_forward(yrtb_projector* h, const float* d_image,
                         const yrtb_events* ev, yrtb_range range, float* d_out,
                         yrtb_stream stream)
{
	if (!d_image || (!d_out && !emptyEvents(ev)))
		return fail(YRTB_ERR_ARGUMENT, "null image or output");
	return dispatchEvents<OP_FWD>(h, ev, range, d_image, d_out, 1.f, 0.f, stream);
}

yrtb_status yrtb_backward(yrtb_projector* h, const float* d_values,
                          const yrtb_events* ev, yrtb_range range,
                          float* d_image, yrtb_stream stream)
{
	if (!d_image || (!d_values && !emptyEvents(ev)))
		return fail(YRTB_ERR_ARGUMENT, "null image or values");
	return dispatchEvents<OP_BWD>(h, ev, range, d_values, d_image, 1.f, 0.f, stream);
}

yrtb_status yrtb_em_step(yrtb_projector* h, const float* d_image, float* d_em,
                         const yrtb_events* ev, yrtb_range range,
                         float global_scale, float denom_threshold,
                         yrtb_stream stream)
{
	if (!d_image || !d_em)
		return fail(YRTB_ERR_ARGUMENT, "null image or EM buffer");
	return dispatchEvents<OP_EM>(h, ev, range, d_image, d_em, global_scale,
	                             denom_threshold, stream);
}

yrtb_status yrtb_em_step_model(yrtb_projector* h, const float* d_image, float* d_em,
                               const yrtb_events* ev, yrtb_range range,
                               float global_scale, float denom_threshold,
                               float* d_model, yrtb_stream stream)
{
	if (!d_image || !d_em || (!d_model && !emptyEvents(ev)))
		return fail(YRTB_ERR_ARGUMENT, "null image, EM buffer or model output");
	return dispatchEvents<OP_EM>(h, ev, range, d_image, d_em, global_scale,
	                             denom_threshold, stream, d_model);
}

yrtb_status yrtb_count_crossings(yrtb_projector* h, const yrtb_events* ev,
                                 yrtb_range range, uint32_t* d_out,
                                 yrtb_stream stream)
{
	if (!d_out && !emptyEvents(ev))
		return fail(YRTB_ERR_ARGUMENT, "null output");
	return dispatchEvents<OP_COUNT>(h, ev, range, nullptr,
	                                reinterpret_cast<float*>(d_out), 1.f, 0.f,
	                                stream);
}

yrtb_status yrtb_trace_walks(yrtb_projector* h, const yrtb_events* ev,
                             yrtb_range range, uint32_t cap, int32_t* d_offsets,
                             float* d_weights, uint32_t* d_counts,
                             yrtb_stream stream)
{
	yrtb_status s = checkEvents(h, ev, range, true);
	if (s != YRTB_OK)
		return s;
	if (range.count == 0)
		return YRTB_OK;
	if (!d_counts || (cap > 0 && (!d_offsets || !d_weights)))
		return fail(YRTB_ERR_ARGUMENT, "null trace output");
	YRTB_CUDA(cudaSetDevice(h->device));
	const Events E = toDev(ev);
	const Range R{range.start, range.stride, range.count};
	cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
	withConfig(h, [&](auto kind, auto tof, auto comp)
	{
		constexpr int K = decltype(kind)::value;
		k_trace<K, decltype(tof)::value, decltype(comp)::value>
		    <<<gridAll(R.count), kBlock, 0, st>>>(h->P, E, R, cap, d_offsets, d_weights,
		                                          d_counts, h->d_err);
	});
	YRTB_LAUNCHED();
	return YRTB_OK;
}

yrtb_status yrtb_attenuation_factors(yrtb_projector* h, const float* d_mu,
                                     const yrtb_image_params* mu_params,
                                     const yrtb_events* ev, yrtb_range range,
                                     float* d_out, yrtb_stream stream)
{
	if (!d_mu || (!d_out && !emptyEvents(ev)) || !validImage(mu_params))
		return fail(YRTB_ERR_ARGUMENT, "invalid attenuation image or output");
	yrtb_status s = checkEvents(h, ev, range, false);
	if (s != YRTB_OK)
		return s;
	if (range.count == 0)
		return YRTB_OK;
	YRTB_CUDA(cudaSetDevice(h->device));
	cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
	const Geom mg = makeGeom(*mu_params);
	int* d_box = nullptr;
	YRTB_CUDA(poolAlloc(&d_box, 6 * sizeof(int), st));
	k_box_init<<<1, 32, 0, st>>>(d_box);
	k_support_box<<<gridFor(mg.nvox, 4), kBlock, 0, st>>>(d_mu, mg, d_box);
	const Range R{range.start, range.stride, range.count};
	const Events E = toDev(ev);
	// Items grouped by walk length: one stable radix pass over an 8-bit
	// bucket keeps the reconstruction order inside each bucket.  Every item's
	// walk is unchanged, so the factors are the same in any order.
	uint8_t *keys = nullptr, *keys2 = nullptr;
	uint32_t *idx = nullptr, *order = nullptr;
	void* temp = nullptr;
	size_t tempBytes = 0;
	const uint64_t n = range.count;
	cudaError_t ce = cudaSuccess;
	if (n < (1ULL << 32))
	{
		ce = poolAlloc(&keys, n, st);
		if (ce == cudaSuccess)
			ce = poolAlloc(&keys2, n, st);
		if (ce == cudaSuccess)
			ce = poolAlloc(&idx, n * sizeof(uint32_t), st);
		if (ce == cudaSuccess)
			ce = poolAlloc(&order, n * sizeof(uint32_t), st);
		if (ce == cudaSuccess)
			ce = cub::DeviceRadixSort::SortPairs(nullptr, tempBytes, keys, keys2, idx, order,
			                                     static_cast<int64_t>(n), 0, 8, st);
		if (ce == cudaSuccess)
			ce = poolAlloc(&temp, tempBytes, st);
		if (ce == cudaSuccess)
		{
			k_att_keys<<<gridFor(n, 16), kBlock, 0, st>>>(h->P, mg, E, R, d_box, keys, idx);
			ce = cub::DeviceRadixSort::SortPairs(temp, tempBytes, keys, keys2, idx, order,
			                                     static_cast<int64_t>(n), 0, 8, st);
		}
	}
	auto release = [&]
	{
		cudaFreeAsync(keys, st);
		cudaFreeAsync(keys2, st);
		cudaFreeAsync(idx, st);
		cudaFreeAsync(order, st);
		cudaFreeAsync(temp, st);
		cudaFreeAsync(d_box, st);
	};
	if (ce != cudaSuccess)
	{
		release();
		return fail(YRTB_ERR_CUDA, std::string("attenuation walk order: ") +
		                               cudaGetErrorString(ce));
	}
	if (h->comp)
		k_attenuation<true><<<gridAll(n), kBlock, 0, st>>>(
		    h->P, mg, E, R, d_mu, d_box, d_out, h->d_err, order);
	else
		k_attenuation<false><<<gridAll(n), kBlock, 0, st>>>(
		    h->P, mg, E, R, d_mu, d_box, d_out, h->d_err, order);
	YRTB_LAUNCHED();
	release();
	return YRTB_OK;
}

yrtb_status yrtb_gather_histo3d(yrtb_projector* h, const float* d_histo,
                                const yrtb_events* ev, yrtb_range range,
                                int invert, float* d_out, yrtb_stream stream)
{
	if (!d_histo || (!d_out && !emptyEvents(ev)))
		return fail(YRTB_ERR_ARGUMENT, "null histogram or output");
	yrtb_status s = checkEvents(h, ev, range, false);
	if (s != YRTB_OK)
		return s;
	if (!h->h3)
		return fail(YRTB_ERR_ARGUMENT, "histogram gather needs detector ids and an even ring");
	if (range.count == 0)
		return YRTB_OK;
	if (!ev->d1)
		return fail(YRTB_ERR_ARGUMENT, "histogram gather needs detector ids and an even ring");
	YRTB_CUDA(cudaSetDevice(h->device));
	k_gather_histo<<<gridAll(range.count), kBlock, 0,
	                 reinterpret_cast<cudaStream_t>(stream)>>>(
	    h->P, h->h3d, toDev(ev), Range{range.start, range.stride, range.count},
	    d_histo, invert, d_out, h->d_err);
	YRTB_LAUNCHED();
	return YRTB_OK;
}

yrtb_status yrtb_sensitivity_histo3d(yrtb_projector* h, float* d_sens,
                                     const float* d_sens_histo,
                                     const float* d_acf_histo,
                                     const float* d_mu,
                                     const yrtb_image_params* mu_params,
                                     int num_subsets, int subset,
                                     yrtb_stream stream)
{
	if (!h || !h->h3)
		return fail(YRTB_ERR_ARGUMENT, "projector has no Histogram3D (odd ring)");
	return dispatchHisto<false>(h, num_subsets, subset, nullptr, d_sens, nullptr,
	                            d_sens_histo, d_acf_histo, nullptr, d_mu,
	                            mu_params, 1.f, 0.f, stream);
}

yrtb_status yrtb_sensitivity_histo3d_crystal(yrtb_projector* h, float* d_sens,
                                             const float* d_crystal_eff,
                                             const float* d_acf_histo,
                                             const float* d_mu,
                                             const yrtb_image_params* mu_params,
                                             int num_subsets, int subset,
                                             yrtb_stream stream)
{
	if (!h || !h->h3)
		return fail(YRTB_ERR_ARGUMENT, "projector has no Histogram3D (odd ring)");
	if (!d_crystal_eff)
		return fail(YRTB_ERR_ARGUMENT, "null crystal factors");
	return dispatchHisto<false>(h, num_subsets, subset, nullptr, d_sens, nullptr,
	                            nullptr, d_acf_histo, nullptr, d_mu, mu_params,
	                            1.f, 0.f, stream, nullptr, 0, d_crystal_eff);
}

yrtb_status yrtb_gather_crystal_product(yrtb_projector* h,
                                        const float* d_crystal_eff,
                                        const yrtb_events* ev, yrtb_range range,
                                        float* d_out, yrtb_stream stream)
{
	if (!d_crystal_eff || (!d_out && !emptyEvents(ev)))
		return fail(YRTB_ERR_ARGUMENT, "null crystal factors or output");
	yrtb_status s = checkEvents(h, ev, range, false);
	if (s != YRTB_OK)
		return s;
	if (range.count == 0)
		return YRTB_OK;
	if (!ev->d1)
		return fail(YRTB_ERR_ARGUMENT, "crystal factors need detector ids");
	YRTB_CUDA(cudaSetDevice(h->device));
	k_gather_crystal<<<gridAll(range.count), kBlock, 0,
	                   reinterpret_cast<cudaStream_t>(stream)>>>(
	    h->P.scan.numDets, toDev(ev), Range{range.start, range.stride, range.count},
	    d_crystal_eff, d_out, h->d_err);
	YRTB_LAUNCHED();
	return YRTB_OK;
}

yrtb_status yrtb_em_step_histo3d(yrtb_projector* h, const float* d_image,
                                 float* d_em, const float* d_meas,
                                 const float* d_sens_histo,
                                 const float* d_acf_histo,
                                 const float* d_add_histo, int num_subsets,
                                 int subset, float global_scale,
                                 float denom_threshold, yrtb_stream stream)
{
	if (!h || !h->h3)
		return fail(YRTB_ERR_ARGUMENT, "projector has no Histogram3D (odd ring)");
	return dispatchHisto<true>(h, num_subsets, subset, d_image, d_em, d_meas,
	                           d_sens_histo, d_acf_histo, d_add_histo, nullptr,
	                           nullptr, global_scale, denom_threshold, stream);
}

yrtb_status yrtb_histo3d_subset_nonzero(yrtb_projector* h, const float* d_meas,
                                        int num_subsets, int subset,
                                        uint64_t* d_k, uint64_t capacity,
                                        uint64_t* n_out, yrtb_stream stream)
{
	if (!h || !h->h3)
		return fail(YRTB_ERR_ARGUMENT, "projector has no Histogram3D (odd ring)");
	if (!d_meas || !d_k || !n_out || num_subsets <= 0 || subset < 0 ||
	    subset >= num_subsets)
		return fail(YRTB_ERR_ARGUMENT, "invalid histogram subset or buffers");
	uint64_t nps = 0;
	const uint64_t count = h3SubsetSize(*h->h3, num_subsets, subset, nps);
	if (capacity < count)
		return fail(YRTB_ERR_ARGUMENT,
		            "bin list capacity " + std::to_string(capacity) +
		                " is below the subset size " + std::to_string(count));
	*n_out = 0;
	if (count == 0)
		return YRTB_OK;
	YRTB_CUDA(cudaSetDevice(h->device));
	cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
	const NonzeroBin pred{h->h3d, d_meas, nps, static_cast<uint64_t>(num_subsets),
	                      static_cast<uint64_t>(subset)};
	const thrust::counting_iterator<uint64_t> first(0);
	unsigned long long* d_num = nullptr;
	void* temp = nullptr;
	size_t tempBytes = 0;
	cudaError_t ce = cub::DeviceSelect::If(nullptr, tempBytes, first, d_k, d_num,
	                                       static_cast<int64_t>(count), pred, st);
	if (ce == cudaSuccess)
		ce = poolAlloc(&d_num, sizeof(unsigned long long), st);
	if (ce == cudaSuccess)
		ce = poolAlloc(&temp, tempBytes, st);
	if (ce == cudaSuccess)
		ce = cub::DeviceSelect::If(temp, tempBytes, first, d_k, d_num,
		                           static_cast<int64_t>(count), pred, st);
	unsigned long long num = 0;
	if (ce == cudaSuccess)
		ce = cudaMemcpyAsync(&num, d_num, sizeof(num), cudaMemcpyDeviceToHost, st);
	cudaFreeAsync(d_num, st);
	cudaFreeAsync(temp, st);
	if (ce == cudaSuccess)
		ce = cudaStreamSynchronize(st);
	if (ce != cudaSuccess)
		return fail(YRTB_ERR_CUDA, std::string("histogram bin selection: ") +
		                               cudaGetErrorString(ce));
	*n_out = num;
	YRTB_LAUNCHED();
	return YRTB_OK;
}

yrtb_status yrtb_em_step_histo3d_list(yrtb_projector* h, const float* d_image,
                                      float* d_em, const float* d_meas,
                                      const float* d_sens_histo,
                                      const float* d_acf_histo,
                                      const float* d_add_histo, int num_subsets,
                                      int subset, const uint64_t* d_k, uint64_t n,
                                      float global_scale, float denom_threshold,
                                      yrtb_stream stream)
{
	if (!h || !h->h3)
		return fail(YRTB_ERR_ARGUMENT, "projector has no Histogram3D (odd ring)");
	if (!d_k && n > 0)
		return fail(YRTB_ERR_ARGUMENT, "null bin list");
	if (n == 0)
		return YRTB_OK;
	return dispatchHisto<true>(h, num_subsets, subset, d_image, d_em, d_meas,
	                           d_sens_histo, d_acf_histo, d_add_histo, nullptr,
	                           nullptr, global_scale, denom_threshold, stream, d_k, n);
}

yrtb_status yrtb_listmode_to_histo3d(yrtb_projector* h, const uint32_t* d1,
                                     const uint32_t* d2, const float* vals,
                                     uint64_t n, float* histo,
                                     uint64_t* n_invalid, yrtb_stream stream)
{
	if (!h || !h->h3 || !d1 || !d2 || !histo)
		return fail(YRTB_ERR_ARGUMENT, "invalid list-mode to histogram arguments");
	YRTB_CUDA(cudaSetDevice(h->device));
	cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
	unsigned long long* d_bad = nullptr;
	YRTB_CUDA(poolAlloc(&d_bad, sizeof(unsigned long long), st));
	YRTB_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(unsigned long long), st));
	if (n > 0)
	{
		k_lm_to_histo<<<gridFor(n, 16), kBlock, 0, st>>>(h->h3d, d1, d2, vals, n,
		                                                 histo, d_bad);
		YRTB_LAUNCHED();
	}
	unsigned long long bad = 0;
	YRTB_CUDA(cudaMemcpyAsync(&bad, d_bad, sizeof(bad), cudaMemcpyDeviceToHost, st));
	YRTB_CUDA(cudaFreeAsync(d_bad, st));
	YRTB_CUDA(cudaStreamSynchronize(st));
	if (n_invalid)
		*n_invalid = bad;
	if (bad > 0)
		return fail(YRTB_ERR_RANGE,
		            std::to_string(bad) +
		                " detector pairs do not respect the maximum ring difference "
		                "or minimum angle difference of the histogram");
	return YRTB_OK;
}

yrtb_status yrtb_unpack_listmode(const void* d_raw, uint64_t n, int has_tof,
                                 int has_randoms, uint32_t num_dets,
                                 uint32_t* d_ts, uint32_t* d_d1, uint32_t* d_d2,
                                 float* d_tof, float* d_randoms,
                                 yrtb_stream stream)
{
	if (!d_raw || !d_d1 || !d_d2)
		return fail(YRTB_ERR_ARGUMENT, "null list-mode buffer");
	if (reinterpret_cast<uintptr_t>(d_raw) % 4 != 0)
		return fail(YRTB_ERR_ARGUMENT, "list-mode records must be 4-byte aligned");
	if (n == 0)
		return YRTB_OK;
	cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
	unsigned long long* d_bad = nullptr;
	YRTB_CUDA(poolAlloc(&d_bad, sizeof(unsigned long long), st));
	YRTB_CUDA(cudaMemsetAsync(d_bad, 0xFF, sizeof(unsigned long long), st));
	const int fields = 3 + (has_tof ? 1 : 0) + (has_randoms ? 1 : 0);
	k_unpack_listmode<<<gridFor(n, 16), kBlock, 0, st>>>(
	    static_cast<const uint32_t*>(d_raw), n, fields, has_tof, has_randoms,
	    num_dets, d_ts, d_d1, d_d2, d_tof, d_randoms, d_bad);
	YRTB_LAUNCHED();
	unsigned long long bad = 0;
	YRTB_CUDA(cudaMemcpyAsync(&bad, d_bad, sizeof(bad), cudaMemcpyDeviceToHost, st));
	YRTB_CUDA(cudaFreeAsync(d_bad, st));
	YRTB_CUDA(cudaStreamSynchronize(st));
	if (bad != ~0ULL)
		return fail(YRTB_ERR_EVENT,
		            "Detectors invalid in list-mode event " + std::to_string(bad));
	return YRTB_OK;
}

yrtb_status yrtb_histo3d_bins(yrtb_projector* h, const uint32_t* d1,
                              const uint32_t* d2, uint64_t n, uint64_t* bins,
                              yrtb_stream stream)
{
	if (!h || !h->h3 || !d1 || !d2 || !bins)
		return fail(YRTB_ERR_ARGUMENT, "invalid histogram map arguments");
	if (n == 0)
		return YRTB_OK;
	YRTB_CUDA(cudaSetDevice(h->device));
	k_bins<<<gridFor(n, 16), kBlock, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
	    h->h3d, d1, d2, n, bins);
	YRTB_LAUNCHED();
	return YRTB_OK;
}

yrtb_status yrtb_histo3d_detpairs(yrtb_projector* h, const uint64_t* bins,
                                  uint64_t n, uint32_t* d1, uint32_t* d2,
                                  yrtb_stream stream)
{
	if (!h || !h->h3 || !d1 || !d2 || !bins)
		return fail(YRTB_ERR_ARGUMENT, "invalid histogram map arguments");
	if (n == 0)
		return YRTB_OK;
	YRTB_CUDA(cudaSetDevice(h->device));
	k_pairs<<<gridFor(n, 16), kBlock, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
	    h->h3d, bins, n, d1, d2);
	YRTB_LAUNCHED();
	return YRTB_OK;
}

yrtb_status yrtb_em_update(float* x, const float* u, const float* s,
                           uint64_t J, int64_t nt, int64_t sens_nt, float thr,
                           const float* scale, yrtb_stream stream)
{
	if (!x || !u || !s || J == 0 || nt <= 0 || (sens_nt != 1 && sens_nt != nt))
		return fail(YRTB_ERR_ARGUMENT, "invalid EM update arguments");
	auto a16 = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
	if (J % 4 == 0 && a16(x) && a16(u) && a16(s))
		k_em_update4<<<gridFor(J / 4, 16), kBlock, 0,
		               reinterpret_cast<cudaStream_t>(stream)>>>(
		    reinterpret_cast<float4*>(x), reinterpret_cast<const float4*>(u),
		    reinterpret_cast<const float4*>(s), J / 4, nt, sens_nt, thr, scale);
	else
		k_em_update<<<gridFor(J, 16), kBlock, 0,
		              reinterpret_cast<cudaStream_t>(stream)>>>(x, u, s, J, nt, sens_nt,
		                                                        thr, scale);
	YRTB_LAUNCHED();
	return YRTB_OK;
}

yrtb_status yrtb_apply_threshold(float* x, const float* m, uint64_t J,
                                 int64_t nt, int broadcast, float thr,
                                 float les, float leo, float gts, float gto,
                                 yrtb_stream stream)
{
	if (!x || !m || J == 0 || nt <= 0)
		return fail(YRTB_ERR_ARGUMENT, "invalid threshold arguments");
	auto a16 = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
	if (J % 4 == 0 && a16(x) && a16(m))
		k_threshold4<<<gridFor(J / 4, 16), kBlock, 0,
		               reinterpret_cast<cudaStream_t>(stream)>>>(
		    reinterpret_cast<float4*>(x), reinterpret_cast<const float4*>(m), J / 4, nt,
		    broadcast, thr, les, leo, gts, gto);
	else
		k_threshold<<<gridFor(J * nt, 16), kBlock, 0,
		              reinterpret_cast<cudaStream_t>(stream)>>>(x, m, J, nt, broadcast,
		                                                        thr, les, leo, gts, gto);
	YRTB_LAUNCHED();
	return YRTB_OK;
}

yrtb_status yrtb_fill(float* x, uint64_t n, float v, yrtb_stream stream)
{
	if (!x)
		return fail(YRTB_ERR_ARGUMENT, "null buffer");
	if (n == 0)
		return YRTB_OK;
	k_fill<<<gridFor(n, 16), kBlock, 0, reinterpret_cast<cudaStream_t>(stream)>>>(x, n, v);
	YRTB_LAUNCHED();
	return YRTB_OK;
}

yrtb_status yrtb_scale(float* x, uint64_t n, float v, yrtb_stream stream)
{
	if (!x)
		return fail(YRTB_ERR_ARGUMENT, "null buffer");
	if (n == 0)
		return YRTB_OK;
	k_scale<<<gridFor(n, 16), kBlock, 0, reinterpret_cast<cudaStream_t>(stream)>>>(x, n, v);
	YRTB_LAUNCHED();
	return YRTB_OK;
}

yrtb_status yrtb_psf_create(const float* kx, int nkx, const float* ky, int nky,
                            const float* kz, int nkz, yrtb_psf** out)
{
	if (!out)
		return fail(YRTB_ERR_ARGUMENT, "null output handle");
	*out = nullptr;
	const float* ks[3] = {kx, ky, kz};
	const int ns[3] = {nkx, nky, nkz};
	for (int a = 0; a < 3; a++)
		if (!ks[a] || ns[a] <= 0 || ns[a] % 2 == 0)
			return fail(YRTB_ERR_ARGUMENT, "Kernel size must be odd");
	auto p = std::make_unique<yrtb_psf>();
	cudaGetDevice(&p->device);
	for (int a = 0; a < 3; a++)
	{
		std::vector<float> f(ks[a], ks[a] + ns[a]);
		std::reverse(f.begin(), f.end());
		p->n[a] = ns[a];
		YRTB_CUDA(cudaMalloc(&p->k[a], ns[a] * sizeof(float)));
		YRTB_CUDA(cudaMalloc(&p->kf[a], ns[a] * sizeof(float)));
		YRTB_CUDA(cudaMemcpy(p->k[a], ks[a], ns[a] * sizeof(float), cudaMemcpyHostToDevice));
		YRTB_CUDA(cudaMemcpy(p->kf[a], f.data(), ns[a] * sizeof(float), cudaMemcpyHostToDevice));
	}
	*out = p.release();
	return YRTB_OK;
}

void yrtb_psf_destroy(yrtb_psf* p)
{
	delete p;
}

yrtb_status yrtb_psf_apply(const yrtb_psf* p, const float* d_in, float* d_out,
                           const yrtb_image_params* ip, int adjoint,
                           float* d_tmp, yrtb_stream stream)
{
	if (!p || !d_in || !d_out || !validImage(ip))
		return fail(YRTB_ERR_ARGUMENT, "invalid PSF arguments");
	if (d_in == d_out)
		return fail(YRTB_ERR_ARGUMENT, "PSF input and output must differ");
	const int dims[3] = {static_cast<int>(ip->nx), static_cast<int>(ip->ny),
	                     static_cast<int>(ip->nz)};
	if ((dims[1] + kPsfBY - 1) / kPsfBY > 65535 ||
	    static_cast<int64_t>(ip->nz) * ip->nt > INT32_MAX)
		return fail(YRTB_ERR_ARGUMENT, "image too large for the PSF launch");
	for (int a = 0; a < 3; a++)
		if (p->n[a] / 2 >= dims[a])
			return fail(YRTB_ERR_ARGUMENT,
			            "PSF kernel half-width must be smaller than the image along each axis");
	YRTB_CUDA(cudaSetDevice(p->device));
	cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
	const uint64_t total = static_cast<uint64_t>(ip->nx) * ip->ny * ip->nz * ip->nt;
	float* tmp = d_tmp;
	if (!tmp)
		YRTB_CUDA(poolAlloc(&tmp, total * sizeof(float), st));
	float* const* k = adjoint ? p->kf : p->k;
	const int planes = static_cast<int>(ip->nz * ip->nt);
	const dim3 block(kPsfBX, kPsfBY);
	const dim3 grid((dims[0] + kPsfBX - 1) / kPsfBX, (dims[1] + kPsfBY - 1) / kPsfBY,
	                std::min((planes + kPsfPlanes - 1) / kPsfPlanes, 65535));
	auto aligned = [](const void* q) { return (reinterpret_cast<uintptr_t>(q) & 15) == 0; };
	const bool vec = dims[0] % 4 == 0 && aligned(d_in) && aligned(d_out) && aligned(tmp);
	// x: in -> out, y: out -> tmp, z: tmp -> out.
	psfPass<0>(grid, block, st, d_in, d_out, dims, planes, k[0], p->n[0], vec);
	psfPass<1>(grid, block, st, d_out, tmp, dims, planes, k[1], p->n[1], vec);
	psfPass<2>(grid, block, st, tmp, d_out, dims, planes, k[2], p->n[2], vec);
	if (!d_tmp)
		YRTB_CUDA(cudaFreeAsync(tmp, st));
	YRTB_LAUNCHED();
	return YRTB_OK;
}

#define YRTB_LR_LAUNCH(KERNEL, ...)                                                        \
	do                                                                                     \
	{                                                                                      \
		const unsigned grid_ = gridFor(J, 8);                                              \
		if (R <= 4)                                                                        \
			KERNEL<4><<<grid_, kBlock, 0, st>>>(__VA_ARGS__);                              \
		else if (R <= 8)                                                                   \
			KERNEL<8><<<grid_, kBlock, 0, st>>>(__VA_ARGS__);                              \
		else if (R <= 16)                                                                  \
			KERNEL<16><<<grid_, kBlock, 0, st>>>(__VA_ARGS__);                             \
		else                                                                               \
			KERNEL<32><<<grid_, kBlock, 0, st>>>(__VA_ARGS__);                             \
	} while (0)

// Vector form: rank <= 16, images of a multiple of 4 voxels, 16-byte aligned.
static bool lrVec(int R, uint64_t J, const void* a, const void* b)
{
	return R <= 16 && J % 4 == 0 && (reinterpret_cast<uintptr_t>(a) & 15) == 0 &&
	       (reinterpret_cast<uintptr_t>(b) & 15) == 0;
}

static yrtb_status lrCheck(int R, int T, uint64_t J)
{
	if (R <= 0 || R > kLrMaxRank)
		return fail(YRTB_ERR_ARGUMENT, "low-rank basis: rank must be in 1..32");
	if (T <= 0 || J == 0)
		return fail(YRTB_ERR_ARGUMENT, "low-rank basis: empty frames or image");
	return YRTB_OK;
}

yrtb_status yrtb_lr_expand(const float* d_W, const float* d_H, int R, int T, uint64_t J,
                           float* d_X, yrtb_stream stream)
{
	if (!d_W || !d_H || !d_X)
		return fail(YRTB_ERR_ARGUMENT, "null low-rank argument");
	yrtb_status s = lrCheck(R, T, J);
	if (s != YRTB_OK)
		return s;
	cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
	if (lrVec(R, J, d_W, d_X))
	{
		const uint64_t J4 = J / 4;
		const unsigned grid_ = gridFor(J4, 8);
		auto W4 = reinterpret_cast<const float4*>(d_W);
		auto X4 = reinterpret_cast<float4*>(d_X);
		if (R <= 4)
			k_lr_expand4<4><<<grid_, kBlock, 0, st>>>(W4, d_H, R, T, J4, X4);
		else if (R <= 8)
			k_lr_expand4<8><<<grid_, kBlock, 0, st>>>(W4, d_H, R, T, J4, X4);
		else
			k_lr_expand4<16><<<grid_, kBlock, 0, st>>>(W4, d_H, R, T, J4, X4);
	}
	else
		YRTB_LR_LAUNCH(k_lr_expand, d_W, d_H, R, T, J, d_X);
	YRTB_LAUNCHED();
	return YRTB_OK;
}

yrtb_status yrtb_lr_contract_w(const float* d_E, const float* d_H, int R, int T, uint64_t J,
                               float* d_Wn, yrtb_stream stream)
{
	if (!d_E || !d_H || !d_Wn)
		return fail(YRTB_ERR_ARGUMENT, "null low-rank argument");
	yrtb_status s = lrCheck(R, T, J);
	if (s != YRTB_OK)
		return s;
	cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
	if (lrVec(R, J, d_E, d_Wn))
	{
		const uint64_t J4 = J / 4;
		const unsigned grid_ = gridFor(J4, 8);
		auto E4 = reinterpret_cast<const float4*>(d_E);
		auto Wn4 = reinterpret_cast<float4*>(d_Wn);
		if (R <= 4)
			k_lr_contract_w4<4><<<grid_, kBlock, 0, st>>>(E4, d_H, R, T, J4, Wn4);
		else if (R <= 8)
			k_lr_contract_w4<8><<<grid_, kBlock, 0, st>>>(E4, d_H, R, T, J4, Wn4);
		else
			k_lr_contract_w4<16><<<grid_, kBlock, 0, st>>>(E4, d_H, R, T, J4, Wn4);
	}
	else
		YRTB_LR_LAUNCH(k_lr_contract_w, d_E, d_H, R, T, J, d_Wn);
	YRTB_LAUNCHED();
	return YRTB_OK;
}

yrtb_status yrtb_lr_contract_h(const float* d_W, const float* d_E, int R, int T, uint64_t J,
                               double* d_Hn, yrtb_stream stream)
{
	if (!d_W || !d_E || !d_Hn)
		return fail(YRTB_ERR_ARGUMENT, "null low-rank argument");
	yrtb_status s = lrCheck(R, T, J);
	if (s != YRTB_OK)
		return s;
	const int P = R * T;
	const size_t smem = static_cast<size_t>(R + T) * (kLrTile + 1) * sizeof(float);
	if (P > kLrPairs * kLrBlock || smem > 227 * 1024)
		return fail(YRTB_ERR_ARGUMENT,
		            "low-rank basis too large for the H contraction "
		            "(rank x frames <= 2048, rank + frames <= 440)");
	cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
	if (smem > 48 * 1024)
		YRTB_CUDA(cudaFuncSetAttribute(k_lr_contract_h,
		                               cudaFuncAttributeMaxDynamicSharedMemorySize,
		                               static_cast<int>(smem)));
	const unsigned blocks = static_cast<unsigned>(std::min<uint64_t>(
	    (J + kLrTile - 1) / kLrTile, static_cast<uint64_t>(gridFor(1 << 30, 2))));
	double* partial = nullptr;
	YRTB_CUDA(poolAlloc(&partial, static_cast<size_t>(blocks) * P * sizeof(double), st));
	k_lr_contract_h<<<blocks, kLrBlock, smem, st>>>(d_W, d_E, R, T, J, partial);
	k_lr_finish<<<(P + kBlock - 1) / kBlock, kBlock, 0, st>>>(partial, blocks, P, d_Hn);
	YRTB_CUDA(cudaFreeAsync(partial, st));
	YRTB_LAUNCHED();
	return YRTB_OK;
}

yrtb_status yrtb_lr_update_h(float* d_H, const double* d_Hn, const float* d_cH, int R, int T,
                             float eps, yrtb_stream stream)
{
	if (!d_H || !d_Hn || !d_cH)
		return fail(YRTB_ERR_ARGUMENT, "null low-rank argument");
	yrtb_status s = lrCheck(R, T, 1);
	if (s != YRTB_OK)
		return s;
	k_lr_update_h<<<(R * T + kBlock - 1) / kBlock, kBlock, 0,
	                reinterpret_cast<cudaStream_t>(stream)>>>(d_H, d_Hn, d_cH, R, T, eps);
	YRTB_LAUNCHED();
	return YRTB_OK;
}

/* Spatially variant PSF (OperatorVarPsf): kernel construction mirrors
 * ConvolutionKernelGaussian / ConvolutionKernelGaussianMixture::setSigmas
 * (src/operators/OperatorVarPsf.cpp:75-240) in FP32 with the host libm. */
yrtb_status yrtb_varpsf_gaussian_kernel(const float* sig, int columns, const float* nstd,
                                        const yrtb_image_params* ip, float* out,
                                        uint64_t cap, int32_t* half_sizes,
                                        uint64_t* size)
{
	if (!sig || !nstd || !validImage(ip) || !half_sizes || !size ||
	    (columns != 3 && columns != 7))
		return fail(YRTB_ERR_ARGUMENT, "invalid Gaussian PSF kernel arguments");
	const float vx = static_cast<float>(ip->length_x / ip->nx);
	const float vy = static_cast<float>(ip->length_y / ip->ny);
	const float vz = static_cast<float>(ip->length_z / ip->nz);
	const bool two = columns == 7;
	if (!(sig[0] > 0.f && sig[1] > 0.f && sig[2] > 0.f) ||
	    (two && !(sig[3] > 0.f && sig[4] > 0.f && sig[5] > 0.f)))
		return fail(YRTB_ERR_ARGUMENT, "Gaussian sigmas must be positive");
	if (two && !(sig[6] >= 0.f && sig[6] <= 1.f))
		return fail(YRTB_ERR_ARGUMENT, "Second Gaussian weight must be in [0, 1]");
	const float sxm = two ? std::max(sig[0], sig[3]) : sig[0];
	const float sym = two ? std::max(sig[1], sig[4]) : sig[1];
	const float szm = two ? std::max(sig[2], sig[5]) : sig[2];
	const int hx = std::max(1, static_cast<int>(std::floor((sxm * nstd[0]) / vx)) - 1);
	const int hy = std::max(1, static_cast<int>(std::floor((sym * nstd[1]) / vy)) - 1);
	const int hz = std::max(1, static_cast<int>(std::floor((szm * nstd[2]) / vz)) - 1);
	half_sizes[0] = hx;
	half_sizes[1] = hy;
	half_sizes[2] = hz;
	const uint64_t n = static_cast<uint64_t>(2 * hx + 1) * (2 * hy + 1) * (2 * hz + 1);
	*size = n;
	if (!out)
		return YRTB_OK;
	if (cap < n)
		return fail(YRTB_ERR_ARGUMENT, "Gaussian PSF kernel buffer too small");
	auto inv2 = [](float s) { return 1.0f / (2 * s * s); };
	const float ix1 = inv2(sig[0]), iy1 = inv2(sig[1]), iz1 = inv2(sig[2]);
	std::vector<float> k(n);
	float sum1 = 0.f, sum2 = 0.f;
	size_t idx = 0;
	for (int dz = -hz; dz <= hz; ++dz)
		for (int dy = -hy; dy <= hy; ++dy)
			for (int dx = -hx; dx <= hx; ++dx, ++idx)
			{
				const float xo = dx * vx, yo = dy * vy, zo = dz * vz;
				const float e1 = -(xo * xo * ix1 + yo * yo * iy1 + zo * zo * iz1);
				k[idx] = std::exp(e1);
				sum1 += k[idx];
				if (two)
				{
					const float e2 = -(xo * xo * inv2(sig[3]) + yo * yo * inv2(sig[4]) +
					                   zo * zo * inv2(sig[5]));
					sum2 += std::exp(e2);
				}
			}
	if (!two)
	{
		for (uint64_t i = 0; i < n; i++)
			out[i] = k[i] / sum1;
		return YRTB_OK;
	}
	if (!(sum1 > 0.f && sum2 > 0.f))
		return fail(YRTB_ERR_ARGUMENT, "2-Gaussian kernel sums must be positive");
	const float w1 = 1.0f - sig[6];
	idx = 0;
	for (int dz = -hz; dz <= hz; ++dz)
		for (int dy = -hy; dy <= hy; ++dy)
			for (int dx = -hx; dx <= hx; ++dx, ++idx)
			{
				const float xo = dx * vx, yo = dy * vy, zo = dz * vz;
				const float e2 = -(xo * xo * inv2(sig[3]) + yo * yo * inv2(sig[4]) +
				                   zo * zo * inv2(sig[5]));
				out[idx] = w1 * k[idx] / sum1 + sig[6] * std::exp(e2) / sum2;
				if (!(out[idx] >= 0.f))
					return fail(YRTB_ERR_ARGUMENT, "2-Gaussian kernel value cannot be negative");
			}
	return YRTB_OK;
}

yrtb_status yrtb_varpsf_create(const float* weights, const int32_t* half_sizes,
                               int num_kernels, const float* range, const float* gap,
                               yrtb_varpsf** out)
{
	if (!out)
		return fail(YRTB_ERR_ARGUMENT, "null output handle");
	*out = nullptr;
	if (!weights || !half_sizes || num_kernels <= 0 || !range || !gap)
		return fail(YRTB_ERR_ARGUMENT, "LUT not defined");
	auto p = std::make_unique<yrtb_varpsf>();
	for (int a = 0; a < 3; a++)
	{
		if (!(gap[a] > 0.f) || !(range[a] >= 0.f))
			return fail(YRTB_ERR_ARGUMENT, "variant PSF ranges and gaps must be positive");
		p->gap[a] = gap[a];
		p->lut[a] = static_cast<int>(std::floor(range[a] / gap[a])) + 1;
	}
	if (static_cast<int64_t>(p->lut[0]) * p->lut[1] * p->lut[2] > num_kernels)
		return fail(YRTB_ERR_ARGUMENT,
		            "variant PSF LUT has fewer kernels than its ranges and gaps need");
	std::vector<int4> meta(num_kernels);
	uint64_t total = 0;
	for (int i = 0; i < num_kernels; i++)
	{
		const int hx = half_sizes[3 * i], hy = half_sizes[3 * i + 1], hz = half_sizes[3 * i + 2];
		if (hx < 0 || hy < 0 || hz < 0)
			return fail(YRTB_ERR_ARGUMENT, "negative PSF kernel half size");
		meta[i] = make_int4(static_cast<int>(total), hx, hy, hz);
		p->maxH[0] = std::max(p->maxH[0], hx);
		p->maxH[1] = std::max(p->maxH[1], hy);
		p->maxH[2] = std::max(p->maxH[2], hz);
		total += static_cast<uint64_t>(2 * hx + 1) * (2 * hy + 1) * (2 * hz + 1);
		if (total > static_cast<uint64_t>(INT32_MAX))
			return fail(YRTB_ERR_ARGUMENT, "variant PSF kernels too large");
	}
	p->numKernels = num_kernels;
	cudaGetDevice(&p->device);
	YRTB_CUDA(cudaMalloc(&p->w, total * sizeof(float)));
	YRTB_CUDA(cudaMalloc(&p->meta, num_kernels * sizeof(int4)));
	YRTB_CUDA(cudaMemcpy(p->w, weights, total * sizeof(float), cudaMemcpyHostToDevice));
	YRTB_CUDA(cudaMemcpy(p->meta, meta.data(), num_kernels * sizeof(int4),
	                     cudaMemcpyHostToDevice));
	*out = p.release();
	return YRTB_OK;
}

void yrtb_varpsf_destroy(yrtb_varpsf* p)
{
	delete p;
}

yrtb_status yrtb_varpsf_apply(const yrtb_varpsf* p, const float* d_in, float* d_out,
                              const yrtb_image_params* ip, int adjoint, yrtb_stream stream)
{
	if (!p || !d_in || !d_out || !validImage(ip))
		return fail(YRTB_ERR_ARGUMENT, "invalid variant PSF arguments");
	if (d_in == d_out)
		return fail(YRTB_ERR_ARGUMENT, "PSF input and output must differ");
	const int dims[3] = {static_cast<int>(ip->nx), static_cast<int>(ip->ny),
	                     static_cast<int>(ip->nz)};
	for (int a = 0; a < 3; a++)
		if (p->maxH[a] >= dims[a])
			return fail(YRTB_ERR_ARGUMENT,
			            "PSF kernel half-width must be smaller than the image along each axis");
	if ((dims[1] + kPsfBY - 1) / kPsfBY > 65535 ||
	    static_cast<int64_t>(ip->nz) * ip->nt > INT32_MAX)
		return fail(YRTB_ERR_ARGUMENT, "image too large for the PSF launch");
	YRTB_CUDA(cudaSetDevice(p->device));
	VarPsfDev P;
	P.w = p->w;
	P.meta = p->meta;
	P.lutX = p->lut[0];
	P.lutY = p->lut[1];
	P.lutZ = p->lut[2];
	P.gapX = p->gap[0];
	P.gapY = p->gap[1];
	P.gapZ = p->gap[2];
	P.vx = static_cast<float>(ip->length_x / ip->nx);
	P.vy = static_cast<float>(ip->length_y / ip->ny);
	P.vz = static_cast<float>(ip->length_z / ip->nz);
	P.cx = ip->nx * P.vx / 2.0f;
	P.cy = ip->ny * P.vy / 2.0f;
	P.cz = ip->nz * P.vz / 2.0f;
	P.maxHx = p->maxH[0];
	P.maxHy = p->maxH[1];
	P.maxHz = p->maxH[2];
	const int planes = static_cast<int>(ip->nz * ip->nt);
	const dim3 block(kPsfBX, kPsfBY);
	// Enough blocks for a few waves; each loops over planes so that the
	// per-block axis tables are built a few thousand times, not per plane.
	const int gx = (dims[0] + kPsfBX - 1) / kPsfBX, gy = (dims[1] + kPsfBY - 1) / kPsfBY;
	const int want = static_cast<int>(gridFor(1u << 30, 16));
	const int gz = std::max(1, std::min(planes, (want + gx * gy - 1) / (gx * gy)));
	const dim3 grid(gx, gy, std::min(gz, 65535));
	cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
	const size_t smem = static_cast<size_t>(dims[0] + dims[1] + dims[2]) * sizeof(int);
	if (smem > 48 * 1024)
		return fail(YRTB_ERR_ARGUMENT, "image too large for the variant PSF (nx + ny + nz > 12288)");
	if (adjoint)
		k_varpsf<true><<<grid, block, smem, st>>>(d_in, d_out, dims[0], dims[1], dims[2], planes, P);
	else
		k_varpsf<false><<<grid, block, smem, st>>>(d_in, d_out, dims[0], dims[1], dims[2], planes, P);
	YRTB_LAUNCHED();
	return YRTB_OK;
}

yrtb_status yrtb_osem_listmode(yrtb_projector* h, const yrtb_events* ev,
                               const float* d_sens, float* d_image,
                               float* d_work, const yrtb_osem_params* p,
                               yrtb_stream stream)
{
	if (!h || !ev || !d_sens || !d_image || !d_work || !p)
		return fail(YRTB_ERR_ARGUMENT, "null OSEM argument");
	if (p->iterations <= 0 || p->subsets <= 0)
		return fail(YRTB_ERR_ARGUMENT, "Not enough OSEM subsets / MLEM iterations");
	YRTB_CUDA(cudaSetDevice(h->device));
	const uint64_t J = static_cast<uint64_t>(h->P.g.nvox);
	const int64_t nt = h->ip.nt;
	float* em = d_work;
	float* sens = d_work + J * nt;
	// With an image-space PSF: the blurred image (also the blurred EM image
	// after the pass) and the PSF's temporary follow.
	float* xpsf = sens + J;
	float* ptmp = xpsf + J * nt;
	// A projector set to YRTB_LAYOUT_TILE_4X2 walks 4 x 2 tiles here too
	// (without an image-space PSF): the image and the sensitivity, given
	// row-major, are converted on entry and the image back on exit, through
	// the EM buffer.
	const bool tile = h->layout == YRTB_LAYOUT_TILE_4X2 && !p->psf && !p->varpsf;
	const int layout = tile ? YRTB_LAYOUT_TILE_4X2 : YRTB_LAYOUT_ROW_MAJOR;
	yrtb_image_params ip1 = h->ip;
	ip1.nt = 1;
	// List-mode sensitivity is shared by all subsets and divided by their
	// number (OSEM::initializeSensImageBuffer, OSEM.cpp:1007-1035).
	yrtb_status s = YRTB_OK;
	if (tile)
	{
		if ((s = yrtb_image_convert_layout(d_sens, sens, &ip1, layout, stream)) != YRTB_OK)
			return s;
	}
	else
	{
		YRTB_CUDA(cudaMemcpyAsync(sens, d_sens, J * sizeof(float),
		                          cudaMemcpyDeviceToDevice,
		                          reinterpret_cast<cudaStream_t>(stream)));
	}
	if (p->subsets != 1)
		s = yrtb_scale(sens, J, 1.0f / static_cast<float>(p->subsets), stream);
	if (s != YRTB_OK)
		return s;
	// x0 = 0.125 (OSEM::INITIAL_VALUE_MLEM), masked where sens <= 0
	// (OSEM_GPU::prepareBuffersForRecon, OSEM_GPU.cu:311-360).
	if (!p->init_from_image)
		if ((s = yrtb_fill(d_image, J * nt, 0.125f, stream)) != YRTB_OK)
			return s;
	if ((s = yrtb_apply_threshold(d_image, d_sens, J, nt, 1, 0.f, 0.f, 0.f, 1.f,
	                              0.f, stream)) != YRTB_OK)
		return s;
	// Converts d_image in place to `to` through the EM buffer.
	auto convertImage = [&](int to) -> yrtb_status
	{
		yrtb_status r = yrtb_image_convert_layout(d_image, em, &h->ip, to, stream);
		if (r != YRTB_OK)
			return r;
		YRTB_CUDA(cudaMemcpyAsync(d_image, em, J * nt * sizeof(float),
		                          cudaMemcpyDeviceToDevice,
		                          reinterpret_cast<cudaStream_t>(stream)));
		return YRTB_OK;
	};
	if (tile && (s = convertImage(YRTB_LAYOUT_TILE_4X2)) != YRTB_OK)
		return s;

	auto subsetOps = [&](int sub) -> yrtb_status
	{
		yrtb_status r;
		if ((r = yrtb_fill(em, J * nt, 0.f, stream)) != YRTB_OK)
			return r;
		yrtb_range range{static_cast<uint64_t>(sub),
		                 static_cast<uint64_t>(p->subsets), 0};
		if (p->subset_offsets)
		{
			range.start = p->subset_offsets[sub];
			range.stride = 1;
			range.count = p->subset_offsets[sub + 1] - p->subset_offsets[sub];
			if (range.count == 0)
				return yrtb_em_update(d_image, em, sens, J, nt, 1, p->em_threshold,
				                      p->d_frame_scale, stream);
		}
		if (p->psf || p->varpsf)
		{
			// OSEM_GPU::computeEMUpdateImage with image PSF
			// (src/recon/OSEM_GPU.cu:456-509): project PSF(x), back-project
			// the ratio, apply PSF^H to the EM image.
			auto blur = [&](const float* in, float* out, int adj)
			{
				return p->psf ? yrtb_psf_apply(p->psf, in, out, &h->ip, adj, ptmp, stream)
				              : yrtb_varpsf_apply(p->varpsf, in, out, &h->ip, adj, stream);
			};
			if ((r = blur(d_image, xpsf, 0)) != YRTB_OK ||
			    (r = yrtb_em_step(h, xpsf, em, ev, range, p->global_scale,
			                      p->denom_threshold, stream)) != YRTB_OK ||
			    (r = blur(em, xpsf, 1)) != YRTB_OK)
				return r;
			return yrtb_em_update(d_image, xpsf, sens, J, nt, 1, p->em_threshold,
			                      p->d_frame_scale, stream);
		}
		if ((r = dispatchEvents<OP_EM>(h, ev, range, d_image, em, p->global_scale,
		                               p->denom_threshold, stream, nullptr, layout)) != YRTB_OK)
			return r;
		return yrtb_em_update(d_image, em, sens, J, nt, 1, p->em_threshold,
		                      p->d_frame_scale, stream);
	};

	cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
	if (!p->use_graph)
	{
		for (int it = 0; it < p->iterations; it++)
			for (int sub = 0; sub < p->subsets; sub++)
				if ((s = subsetOps(sub)) != YRTB_OK)
					return s;
		return tile ? convertImage(YRTB_LAYOUT_ROW_MAJOR) : YRTB_OK;
	}
	// One graph per subset, captured once and replayed every iteration.
	if (st == nullptr)
		return fail(YRTB_ERR_ARGUMENT, "CUDA-graph OSEM needs a non-default stream");
	std::vector<cudaGraphExec_t> execs(p->subsets, nullptr);
	auto cleanup = [&]
	{
		for (auto& e : execs)
			if (e)
				cudaGraphExecDestroy(e);
	};
	for (int sub = 0; sub < p->subsets; sub++)
	{
		cudaGraph_t g = nullptr;
		cudaError_t ce = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
		if (ce != cudaSuccess)
		{
			cleanup();
			return fail(YRTB_ERR_CUDA, cudaGetErrorString(ce));
		}
		const yrtb_status r = subsetOps(sub);
		ce = cudaStreamEndCapture(st, &g);
		if (r != YRTB_OK || ce != cudaSuccess)
		{
			if (g)
				cudaGraphDestroy(g);
			cleanup();
			return r != YRTB_OK ? r : fail(YRTB_ERR_CUDA, cudaGetErrorString(ce));
		}
		ce = cudaGraphInstantiate(&execs[sub], g, 0);
		cudaGraphDestroy(g);
		if (ce != cudaSuccess)
		{
			cleanup();
			return fail(YRTB_ERR_CUDA, cudaGetErrorString(ce));
		}
	}
	for (int it = 0; it < p->iterations; it++)
		for (int sub = 0; sub < p->subsets; sub++)
		{
			const cudaError_t ce = cudaGraphLaunch(execs[sub], st);
			if (ce != cudaSuccess)
			{
				cleanup();
				return fail(YRTB_ERR_CUDA, cudaGetErrorString(ce));
			}
		}
	cleanup();
	return tile ? convertImage(YRTB_LAYOUT_ROW_MAJOR) : YRTB_OK;
}

yrtb_status yrtb_autotune(yrtb_projector* h, const float* d_image,
                          const yrtb_events* ev, int num_subsets,
                          uint64_t max_sample, yrtb_tune_report* report,
                          yrtb_stream stream)
{
	if (!h || !d_image || !ev || !report || num_subsets <= 0)
		return fail(YRTB_ERR_ARGUMENT, "invalid autotune arguments");
	*report = yrtb_tune_report{};
	report->best = h->launch;
	if (h->kind != K_SIDDON && h->kind != K_SIDDON_MR)
		return YRTB_OK;
	const bool multiRay = h->kind == K_SIDDON_MR;
	yrtb_range all{0, 1, 0};
	yrtb_status s = checkEvents(h, ev, all, true);
	if (s != YRTB_OK)
		return s;
	const uint64_t S = static_cast<uint64_t>(num_subsets);
	uint64_t n = ev->count == 0 ? 0 : (ev->count + S - 1) / S;  // subset 0
	if (max_sample > 0 && n > max_sample)
		n = max_sample;
	if (n == 0)
		return YRTB_OK;
	YRTB_CUDA(cudaSetDevice(h->device));
	cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);

	// Temporaries: the sample twice (as drawn, and ordered per candidate),
	// two permutations, one EM image.
	std::vector<void*> bufs;
	auto release = [&]
	{
		for (void* b : bufs)
			cudaFreeAsync(b, st);
		bufs.clear();
	};
	auto alloc = [&](size_t bytes, void** out) -> bool
	{
		*out = nullptr;
		if (poolAlloc(out, bytes, st) != cudaSuccess)
			return false;
		bufs.push_back(*out);
		return true;
	};
	yrtb_events A = *ev, B = *ev;
	A.count = B.count = n;
	bool ok = true;
	auto twin = [&](const void* src, size_t width, const void** a, const void** b)
	{
		if (!src || !ok)
			return;
		void *pa = nullptr, *pb = nullptr;
		ok = alloc(n * width, &pa) && alloc(n * width, &pb);
		*a = pa;
		*b = pb;
	};
	twin(ev->d1, 4, reinterpret_cast<const void**>(&A.d1), reinterpret_cast<const void**>(&B.d1));
	twin(ev->d2, 4, reinterpret_cast<const void**>(&A.d2), reinterpret_cast<const void**>(&B.d2));
	twin(ev->lor, 24, reinterpret_cast<const void**>(&A.lor), reinterpret_cast<const void**>(&B.lor));
	twin(ev->orient, 24, reinterpret_cast<const void**>(&A.orient), reinterpret_cast<const void**>(&B.orient));
	twin(ev->tof_ps, 4, reinterpret_cast<const void**>(&A.tof_ps), reinterpret_cast<const void**>(&B.tof_ps));
	twin(ev->frame, 4, reinterpret_cast<const void**>(&A.frame), reinterpret_cast<const void**>(&B.frame));
	twin(ev->motion_frame, 4, reinterpret_cast<const void**>(&A.motion_frame), reinterpret_cast<const void**>(&B.motion_frame));
	twin(ev->measurement, 4, reinterpret_cast<const void**>(&A.measurement), reinterpret_cast<const void**>(&B.measurement));
	twin(ev->sens, 4, reinterpret_cast<const void**>(&A.sens), reinterpret_cast<const void**>(&B.sens));
	twin(ev->att, 4, reinterpret_cast<const void**>(&A.att), reinterpret_cast<const void**>(&B.att));
	twin(ev->additive, 4, reinterpret_cast<const void**>(&A.additive), reinterpret_cast<const void**>(&B.additive));
	void *perm = nullptr, *perm2 = nullptr, *em = nullptr;
	const uint64_t J = static_cast<uint64_t>(h->P.g.nvox) * h->ip.nt;
	ok = ok && alloc(n * 8, &perm) && alloc(n * 8, &perm2) && alloc(J * 4, &em);
	if (!ok)
	{
		release();
		return fail(YRTB_ERR_CUDA, "autotune: device allocation failed");
	}
	// Sample = events 0, S, 2S, ... (subset 0 of the interleaved subsets).
	k_iota_stride<<<gridFor(n, 8), kBlock, 0, st>>>(
	    static_cast<unsigned long long*>(perm), n, S);
	yrtb_events src = *ev;
	src.count = n;
	if ((s = gatherEvents(&src, static_cast<uint64_t*>(perm), &A, stream, false)) != YRTB_OK)
	{
		release();
		return s;
	}
	cudaMemsetAsync(em, 0, J * 4, st);

	const yrtb_launch_config saved = h->launch;
	cudaEvent_t e0 = nullptr, e1 = nullptr;
	cudaEventCreate(&e0);
	cudaEventCreate(&e1);
	const yrtb_range r{0, 1, n};
	int bestIdx = -1;
	// Orders the sample for c (unless it is ordered so already) and times the
	// EM step with c: best of 3 after one warm-up.
	yrtb_launch_config ordered{};
	bool haveOrder = false;
	auto timeOne = [&](const yrtb_launch_config& c) -> yrtb_status
	{
		if (report->num_tried >= YRTB_TUNE_MAX)
			return YRTB_OK;
		yrtb_status q;
		if (!haveOrder || c.bucket_shift != ordered.bucket_shift ||
		    c.order != ordered.order || c.tile_shift != ordered.tile_shift)
		{
			if ((q = orderEvents(h, &A, 1, c, static_cast<uint64_t*>(perm2), st)) != YRTB_OK ||
			    (q = yrtb_events_gather(&A, static_cast<uint64_t*>(perm2), &B, stream)) != YRTB_OK)
				return q;
			ordered = c;
			haveOrder = true;
		}
		h->launch = c;
		float best = 3.4e38f;
		for (int rep = 0; rep < 4; rep++)
		{
			cudaEventRecord(e0, st);
			q = yrtb_em_step(h, d_image, static_cast<float*>(em), &B, r, 1.f, 1e-35f, stream);
			cudaEventRecord(e1, st);
			const cudaError_t ce = cudaEventSynchronize(e1);
			if (q != YRTB_OK)
				return q;
			if (ce != cudaSuccess)
				return fail(YRTB_ERR_CUDA, cudaGetErrorString(ce));
			float ms = 0.f;
			if (rep > 0 && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess)
				best = std::min(best, ms);  // rep 0 warms up
		}
		const int i = report->num_tried++;
		report->tried[i] = c;
		report->ms[i] = best;
		if (bestIdx < 0 || best < report->ms[bestIdx])
			bestIdx = i;
		return YRTB_OK;
	};
	// Stage 1: event orders x vector groups, with the current block size and
	// threads per LOR (one thread per LOR when the projector splits none; a
	// multi-ray projector keeps its lanes per event and tries the register
	// float4 and the pair reductions, the vector modes its walks use).
	const int orders[3][2] = {{YRTB_ORDER_LOR, 1}, {YRTB_ORDER_SPATIAL, 1},
	                          {YRTB_ORDER_SPATIAL, 2}};
	for (int shift : {3, 4, 5})
		for (const auto& ot : orders)
			for (int vec : {2, 8, 4, 1, 0})
			{
				if (multiRay && (vec == 4 || vec == 1))
					continue;
				yrtb_launch_config c = saved;
				c.threads_per_lor = multiRay ? saved.threads_per_lor : 1;
				c.bucket_shift = shift;
				c.order = ot[0];
				c.tile_shift = ot[1];
				c.vector_groups = vec;
				if (s == YRTB_OK)
					s = timeOne(c);
			}
	// Stage 2: block size x threads per LOR on the fastest order.
	if (s == YRTB_OK && bestIdx >= 0)
	{
		const yrtb_launch_config o = report->tried[bestIdx];
		const bool split = h->comp && !h->det;
		const int lanes = rayLanes(h->P.numRays);
		for (int block : {128, 256})
			for (int tpl : {1, 2, 4, 8})
			{
				if (multiRay)
				{
					// Multi-ray: 256-thread blocks; one thread per event or one
					// lane per ray.
					if (block != 256 || h->det || (tpl != 1 && tpl != lanes))
						continue;
				}
				else if (tpl == 8 || (tpl > 1 && (!split || h->layout == YRTB_LAYOUT_TILE_4X2)) ||
				         (h->det && (block != 256 || tpl != 1)))
					continue;
				if (block == o.block && tpl == o.threads_per_lor)
					continue;
				yrtb_launch_config c = o;
				c.block = block;
				c.threads_per_lor = tpl;
				if (s == YRTB_OK)
					s = timeOne(c);
			}
	}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	release();
	h->launch = bestIdx >= 0 ? report->tried[bestIdx] : saved;
	report->best = h->launch;
	report->sample_events = n;
	if (s != YRTB_OK)
		return s;
	YRTB_LAUNCHED();
	return YRTB_OK;
}

}  // extern "C"

// ------------------------------------------- OSEM without any allocation --
// Scratch of yrtb_osem_listmode_static: the EM image (nt frames) followed by
// the 1/numSubsets-scaled sensitivity image.  A file-scope device array, so
// the entry point never allocates; every GPU that loads the library holds it
// (16 MiB) until the process exits.
static __device__ __align__(256) float g_osemStaticScratch[YRTB_OSEM_STATIC_MAX_FLOATS];

namespace
{
// Device address of g_osemStaticScratch on the current device.  In host code
// the array's name is only a host-side stand-in, so the address is looked up
// with the device current, on every call: the lookup allocates nothing once
// the module is loaded, and an address kept from before a device reset would
// point into a context that no longer exists.
yrtb_status osemStaticScratch(float** out)
{
	void* p = nullptr;
	const cudaError_t e = cudaGetSymbolAddress(&p, g_osemStaticScratch);
	if (e != cudaSuccess || p == nullptr)
		return fail(YRTB_ERR_CUDA,
		            std::string("cudaGetSymbolAddress(osem static scratch): ") +
		                cudaGetErrorString(e));
	*out = static_cast<float*>(p);
	return YRTB_OK;
}
}  // namespace

extern "C" yrtb_status yrtb_osem_listmode_static(yrtb_projector* h,
                                                 const yrtb_events* ev,
                                                 const float* d_sens,
                                                 float* d_image,
                                                 const yrtb_osem_params* p,
                                                 yrtb_stream stream)
{
	if (!h || !ev || !d_sens || !d_image || !p)
		return fail(YRTB_ERR_ARGUMENT, "null OSEM argument");
	if (p->use_graph)
		return fail(YRTB_ERR_ARGUMENT,
		            "yrtb_osem_listmode_static does not build CUDA graphs "
		            "(instantiating one allocates); set use_graph = 0");
	const uint64_t J = static_cast<uint64_t>(h->P.g.nvox);
	const uint64_t need = J * static_cast<uint64_t>(h->ip.nt) + J +
	                      ((p->psf || p->varpsf) ? 2 * J * static_cast<uint64_t>(h->ip.nt) : 0);
	if (need > YRTB_OSEM_STATIC_MAX_FLOATS)
		return fail(YRTB_ERR_ARGUMENT,
		            "image too large for yrtb_osem_listmode_static: needs " +
		                std::to_string(need) + " floats of scratch ((nt+1) x voxels "
		                "without an image-space PSF, (3nt+1) x voxels with one), "
		                "the static buffer holds " +
		                std::to_string(static_cast<uint64_t>(YRTB_OSEM_STATIC_MAX_FLOATS)) +
		                "; use yrtb_osem_listmode with a caller-provided work buffer");
	YRTB_CUDA(cudaSetDevice(h->device));
	float* scratch = nullptr;
	const yrtb_status st = osemStaticScratch(&scratch);
	if (st != YRTB_OK)
		return st;
	// The shared driver overwrites the sensitivity part and clears the EM
	// image before every subset, so stale contents of earlier calls are never
	// read.
	return yrtb_osem_listmode(h, ev, d_sens, d_image, scratch, p, stream);
}
