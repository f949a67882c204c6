// Device-side projection math for libyrtb (sm_100a).
//
// This translation unit is compiled with -fmad=false: in YRTB_MIRROR mode
// every expression below is evaluated in FP32 with the operation order of the
// reference CPU projector, so the voxel index sequence of each ray (and, for
// non-TOF rays, every weight) is bit-identical to it.  The traversal itself
// is written from the published incremental Siddon method: parametric entry
// into the image slabs, then stepping to the nearest of the next x/y/z plane
// crossings.  Reference behaviour followed (paths inside yrt-pet):
//   FOV-cylinder clip, slab alphas, entry step, tie rule (<=), early exit
//                                 src/operators/ProjectorSiddon.cpp:495-766
//   TOF window and midpoint weight include/yrt-pet/operators/TimeOfFlight.hpp:53-84
//   multi-ray offsets (curand)    include/yrt-pet/operators/SiddonKernels.cuh:27-84
//   distance-driven footprint     src/operators/ProjectorDD.cpp:260-578
//   projection-space PSF integral include/yrt-pet/operators/ProjectorUtils.hpp:43-98
#pragma once

#include <cuda_runtime.h>
#include <curand_kernel.h>
#include <stdint.h>

#include <type_traits>

namespace yrtb
{

constexpr double kSpeedOfLightMmPs = 0.299792458;
// The reference stores c as a double holding the float value 0.299792458f.
constexpr double kSpeedOfLightMmPsFlt = 0.299792458f;

struct Geom
{
	int nx, ny, nz, nt;
	int64_t nxy, nvox;
	float lx, ly, lz;
	float vx, vy, vz;
	float fovRadius;
	float offx, offy, offz;
};

struct TofP
{
	float sigma, trunc, norm;
};

struct Psf
{
	const float* taps;     // num_s * size
	const float* flipped;  // adjoint taps
	int num_s, size;
	float sStep, kSpacing;
	// Prefix sums of the trapezoid bins of each kernel row (num_s * (size +
	// 3)): prefix[m] = sum over bins xi = -1 .. m-2 of step (v(xi) + v(xi+1)) / 2.
	const float* prefix;
	const float* prefixFlipped;
};

struct Scan
{
	const float4* pos;  // crystal centres
	const float4* ori;  // crystal orientations
	uint32_t numDets;
	float crystalZ, crystalTrans;
};

// Device copy of the event arrays (see yrtb_events in include/yrt_b200.h).
struct Events
{
	const uint32_t* d1;
	const uint32_t* d2;
	const float* lor;
	const float* tof;
	const int32_t* frame;
	const int32_t* mframe;
	const float* motion;
	uint64_t numMotion;
	const float* meas;
	const float* sens;
	const float* att;
	const float* add;
	// EM step only: when not null, each event's model value (forward
	// projection with its corrections, the denominator of the EM ratio) is
	// written here; 0 for an event that is skipped.
	float* model;
	// With lor: crystal orientations n1, n2 (6 floats per event), or null.
	const float* orient;
};

struct Range
{
	uint64_t start, stride, count;
};

__device__ __forceinline__ float3 f3sub(float3 a, float3 b)
{
	return make_float3(a.x - b.x, a.y - b.y, a.z - b.z);
}

// ---------------------------------------------------------------- TOF ----
// Alpha window of the TOF kernel: 0.5 + (c*t/2 -/+ trunc)/L clamped to [0,1],
// with the reference's float/double mix.
__device__ __forceinline__ void tofAlphaRange(const TofP& t, float lorNorm,
                                              float tof_ps, float& amin,
                                              float& amax)
{
	if (t.trunc <= 0.f)
	{
		amin = 0.f;
		amax = 1.f;
		return;
	}
	const float tof_mm =
	    static_cast<float>(static_cast<double>(tof_ps) * kSpeedOfLightMmPsFlt * 0.5);
	amin = static_cast<float>(fmax(0.0, 0.5 + static_cast<double>((tof_mm - t.trunc) / lorNorm)));
	amax = static_cast<float>(fmin(1.0, 0.5 + static_cast<double>((tof_mm + t.trunc) / lorNorm)));
}

// Centre of the TOF kernel in mm from p1: L/2 + c*t/2, with the reference's
// float/double mix.
__device__ __forceinline__ float tofCenter(float lorNorm, float tof_ps)
{
	const float tof_mm =
	    static_cast<float>(static_cast<double>(tof_ps) * kSpeedOfLightMmPsFlt * 0.5);
	return static_cast<float>(0.5 * static_cast<double>(lorNorm) +
	                          static_cast<double>(tof_mm));
}

// Gaussian TOF weight evaluated at the centre of [lo, hi] (mm along the LOR).
__device__ __forceinline__ float tofWeight(const TofP& t, float lorNorm,
                                           float tof_ps, float lo, float hi)
{
	const float pc = tofCenter(lorNorm, tof_ps);
	const float xc = (0.5f * (lo + hi) - pc) / t.sigma;
	return expf(-0.5f * xc * xc) * t.norm;
}

// Parametric interval of a ray inside the slab [r0, r1] along one axis.
template <typename R>
__device__ __forceinline__ void slabAlpha(R r0, R r1, R p1, R p2, R inv,
                                          R& amin, R& amax)
{
	amin = R(0);
	amax = R(1);
	if (p1 != p2)
	{
		const R a0 = (r0 - p1) * inv;
		const R a1 = (r1 - p1) * inv;
		if (a0 < a1)
		{
			amin = a0;
			amax = a1;
		}
		else
		{
			amin = a1;
			amax = a0;
		}
	}
	else if (p1 < r0 || p1 > r1)
	{
		amax = R(0);
		amin = R(1);
	}
}

// ------------------------------------------------------------ Siddon ----
// Walks one ray through the image grid and calls visit(offset, weight) for
// each voxel crossing, in order.  p1, p2: endpoints relative to the image
// centre.  COMP chooses the first planes in FP64 and takes the entry voxel
// from the walk's plane bookkeeping (see begin); the parametric set-up and
// the walk are FP32 in both modes.
//
// The walk is a state machine: begin() sets up the ray and finds its first
// non-empty segment, emitFirst() visits it, next() takes one step.
// siddonWalk() runs it to the end on one thread; siddonWalkWarp() runs the
// rays of a whole warp in lock step.
//
// TILE: the image is stored in tiles of 4 x 2 voxels (x, y) of one z plane,
// 8 floats (one 32-byte sector) per tile, tiles in row-major order inside a
// plane and planes in z order (tileOffset); nx a multiple of 4, ny of 2.  An
// aligned group of four floats is then a 2 x 2 square instead of 4 voxels of
// one row, so that a ray crossing the plane in any direction stays longer in
// one group and one sector.  Same voxels, weights and order: only the
// offsets change.
__device__ __forceinline__ int tileOffset(int vx, int vy, int vz, int nx, int nxy)
{
	return vz * nxy + (vy >> 1) * (2 * nx) + ((vx >> 2) << 3) + (((vx >> 1) & 1) << 2) +
	       ((vy & 1) << 1) + (vx & 1);
}

template <bool TOF, bool COMP, bool TILE = false>
struct SiddonWalker
{
	float3 p1, p2;
	float inv_x, inv_y, inv_z;
	float fdx, fdy, fdz;
	int dir_x, dir_y, dir_z;
	float d_norm, amax;
	float a_cur, a_next;
	float x_cur, y_cur, z_cur, ax_next, ay_next, az_next;
	bool sx, sy, sz;
	int step, maxSteps;
	// COMP: linear voxel index moved by a per-step delta.
	int lin, dprev, dny, dnz;
	unsigned nvox;
	// COMP and TILE: parity of the voxel's x and y, and the offset deltas of
	// one x / y step from an odd or an even coordinate in the ray's direction.
	int px, py, dxo, dxe, dyo, dye;
	// Mirror: voxel coordinates and row offset, as the reference keeps them.
	int vx, vy, vz, off, dir_prev, nx, ny, nz, nxy;
	// TOF weight constants.
	float pc, sigma, norm, hs, pcs, dnn;

	// Advances to the nearest crossing; ties step together (<= on the
	// crossing values from the start of the step, i.e. every axis whose
	// crossing equals the minimum).  Written with selects instead of
	// branches so that the threads of a warp, whose rays step along
	// different axes, stay converged; every value is the one the branchy
	// formulation computes.  Each axis's next crossing is recomputed as
	// (plane - p1) * inv whether it stepped or not: an axis that did not
	// step keeps its plane, so the product has the bits it had (the first
	// crossing is that product too), and no select of the old value is
	// needed.  An axis the ray runs parallel to has inv = +inf and a plane
	// above p1, so its crossing stays +inf.
	__device__ __forceinline__ void advance()
	{
		const float ax = ax_next, ay = ay_next, az = az_next;
		const float m = fminf(fminf(ax, ay), az);
		sx = ax == m;
		sy = ay == m;
		sz = az == m;
		x_cur = sx ? x_cur + fdx : x_cur;
		y_cur = sy ? y_cur + fdy : y_cur;
		z_cur = sz ? z_cur + fdz : z_cur;
		ax_next = (x_cur - p1.x) * inv_x;
		ay_next = (y_cur - p1.y) * inv_y;
		az_next = (z_cur - p1.z) * inv_z;
		a_next = fminf(m, amax);
	}

	template <typename Visit>
	__device__ __forceinline__ void emit(int o, Visit& visit)
	{
		float w;
		if constexpr (TOF && COMP)
		{
			// Compensated TOF weight, per segment [a, b]:
			//   (b - a) * L * norm * 2^(-y^2),  y = x sqrt(log2(e) / 2),
			//   x = ((a + b) L/2 - pc) / sigma
			// with y = (a + b) * hs - pcs in one fused multiply-add (the
			// constant folded into hs and pcs) and the hardware base-2
			// exponential (relative error below 2^-21).
			const float y = __fmaf_rn(a_cur + a_next, hs, -pcs);
			float g2;
			asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(g2) : "f"(-(y * y)));
			w = (a_next - a_cur) * dnn * g2;
		}
		else
		{
			w = (a_next - a_cur) * d_norm;
		}
		if constexpr (TOF && !COMP)
		{
			// The reference's expression order (TimeOfFlight.hpp:74-84).
			const float lo = a_cur * d_norm, hi = a_next * d_norm;
			const float xc = (0.5f * (lo + hi) - pc) / sigma;
			w *= expf(-0.5f * xc * xc) * norm;
		}
		visit(o, w);
		a_cur = a_next;
	}

	// Sets up the ray and finds its first non-empty segment; false if the
	// ray has nothing to visit.
	__device__ __forceinline__ bool begin(const Geom& g, const float3 q1,
	                                      const float3 q2, const TofP& tp,
	                                      float tofValue, float wlo, float whi,
	                                      int part, int parts)
	{
		p1 = q1;
		p2 = q2;
		// 1. Clip to the FOV cylinder.
		float t0, t1;
		{
			const float A = (p2.x - p1.x) * (p2.x - p1.x) + (p2.y - p1.y) * (p2.y - p1.y);
			const float B = 2.0f * ((p2.x - p1.x) * p1.x + (p2.y - p1.y) * p1.y);
			const float C = p1.x * p1.x + p1.y * p1.y - g.fovRadius * g.fovRadius;
			const float Delta = B * B - 4.0f * A * C;
			if (A != 0.0f)
			{
				if (Delta <= 0.0f)
					return false;
				const float sq = sqrtf(Delta);
				t0 = (-B - sq) / (2.0f * A);
				t1 = (-B + sq) / (2.0f * A);
			}
			else
			{
				t0 = 0.f;
				t1 = 1.f;
			}
		}
		const float3 d12 = f3sub(p1, p2);
		d_norm = sqrtf(d12.x * d12.x + d12.y * d12.y + d12.z * d12.z);
		const bool flat_x = (p1.x == p2.x);
		const bool flat_y = (p1.y == p2.y);
		const bool flat_z = (p1.z == p2.z);
		inv_x = flat_x ? 0.0f : 1.0f / (p2.x - p1.x);
		inv_y = flat_y ? 0.0f : 1.0f / (p2.y - p1.y);
		inv_z = flat_z ? 0.0f : 1.0f / (p2.z - p1.z);
		dir_x = (inv_x >= 0.0f) ? 1 : -1;
		dir_y = (inv_y >= 0.0f) ? 1 : -1;
		dir_z = (inv_z >= 0.0f) ? 1 : -1;

		// 2. Intersection with the volume.
		const float dx = g.vx, dy = g.vy, dz = g.vz;
		const float inv_dx = 1.0f / dx, inv_dy = 1.0f / dy, inv_dz = 1.0f / dz;
		const float x0 = -g.lx * 0.5f, x1 = g.lx * 0.5f;
		const float y0 = -g.ly * 0.5f, y1 = g.ly * 0.5f;
		const float z0 = -g.lz * 0.5f, z1 = g.lz * 0.5f;
		float amin;
		{
			float ax_min, ay_min, az_min, ax_max, ay_max, az_max;
			slabAlpha<float>(-0.5f * g.lx, 0.5f * g.lx, p1.x, p2.x, inv_x, ax_min, ax_max);
			slabAlpha<float>(-0.5f * g.ly, 0.5f * g.ly, p1.y, p2.y, inv_y, ay_min, ay_max);
			slabAlpha<float>(-0.5f * g.lz, 0.5f * g.lz, p1.z, p2.z, inv_z, az_min, az_max);
			// max/min over {0|1, t, ax, ay, az} in the reference's order.
			amin = fmaxf(fmaxf(fmaxf(fmaxf(0.0f, t0), ax_min), ay_min), az_min);
			amax = fminf(fminf(fminf(fminf(1.0f, t1), ax_max), ay_max), az_max);
		}
		if constexpr (TOF)
		{
			float a0, a1;
			tofAlphaRange(tp, d_norm, tofValue, a0, a1);
			amin = fmaxf(amin, a0);
			amax = fminf(amax, a1);
		}
		// Optional extra window [wlo, whi] (defaults leave amin, amax unchanged).
		amin = fmaxf(amin, wlo);
		amax = fminf(amax, whi);
		if (parts > 1)
		{
			// Piece `part` of `parts` (several threads per LOR).  The cuts sit
			// on voxel planes of the axis the ray crosses most often, so every
			// segment of the walk stays whole and keeps the TOF weight of its
			// midpoint; neighbouring pieces compute the same cut bit for bit.
			const float cx = flat_x ? -1.f : fabsf(p2.x - p1.x) * inv_dx;
			const float cy = flat_y ? -1.f : fabsf(p2.y - p1.y) * inv_dy;
			const float cz = flat_z ? -1.f : fabsf(p2.z - p1.z) * inv_dz;
			const int ax = (cx >= cy && cx >= cz) ? 0 : (cy >= cz ? 1 : 2);
			const float q1a = ax == 0 ? p1.x : (ax == 1 ? p1.y : p1.z);
			const float q2a = ax == 0 ? p2.x : (ax == 1 ? p2.y : p2.z);
			const float qi = ax == 0 ? inv_x : (ax == 1 ? inv_y : inv_z);
			const float q0 = ax == 0 ? x0 : (ax == 1 ? y0 : z0);
			const float dq = ax == 0 ? dx : (ax == 1 ? dy : dz);
			const float lo = amin, span = amax - amin;
			auto cut = [&](int j) -> float
			{
				const float at = lo + (static_cast<float>(j) / static_cast<float>(parts)) * span;
				const float plane = q0 + rintf((q1a + at * (q2a - q1a) - q0) / dq) * dq;
				return fminf(fmaxf((plane - q1a) * qi, lo), lo + span);
			};
			const float hi = amax;
			amin = part == 0 ? lo : cut(part);
			amax = part == parts - 1 ? hi : cut(part + 1);
		}

		a_cur = amin;
		a_next = -1.0f;
		x_cur = (inv_x > 0.0f) ? x0 : x1;
		y_cur = (inv_y > 0.0f) ? y0 : y1;
		z_cur = (inv_z > 0.0f) ? z0 : z1;
		if ((inv_x >= 0.0f && p1.x > x1) || (inv_x < 0.0f && p1.x < x0) ||
		    (inv_y >= 0.0f && p1.y > y1) || (inv_y < 0.0f && p1.y < y0) ||
		    (inv_z >= 0.0f && p1.z > z1) || (inv_z < 0.0f && p1.z < z0))
			return false;

		// First plane crossing at or beyond the entry point, per axis: the
		// plane index is ceil of the entry position's distance from the
		// walk's start plane in voxels, in FP32 as the reference computes it,
		// or in FP64 (COMP) so that an entry within float rounding of a plane
		// cannot skip that plane.
		auto firstPlane = [&](float q1a, float q2a, float inv, int dir, float d,
		                      float& cur) -> float
		{
			long long k;
			if constexpr (COMP)
				k = static_cast<long long>(
				    ceil(double(dir) * (double(a_cur) * (double(q2a) - double(q1a)) -
				                        double(cur) + double(q1a)) * (1.0 / double(d))));
			else
				k = static_cast<long long>(
				    ceilf(static_cast<float>(dir) * (a_cur * (q2a - q1a) - cur + q1a) / d));
			cur += static_cast<float>(k * dir) * d;
			return (cur - q1a) * inv;
		};
		ax_next = flat_x ? 3.402823466e+38f : firstPlane(p1.x, p2.x, inv_x, dir_x, dx, x_cur);
		ay_next = flat_y ? 3.402823466e+38f : firstPlane(p1.y, p2.y, inv_y, dir_y, dy, y_cur);
		az_next = flat_z ? 3.402823466e+38f : firstPlane(p1.z, p2.z, inv_z, dir_z, dz, z_cur);
		// Parallel axes: crossings at +inf from here on (advance), planes one
		// voxel above p1 (their direction is +1), which no step brings back.
		// Both compare above every crossing of the other axes and above
		// amax <= 1, as the FLT_MAX above does.
		{
			const float inf = __int_as_float(0x7f800000);
			if (flat_x)
			{
				inv_x = inf;
				x_cur = p1.x + dx;
			}
			if (flat_y)
			{
				inv_y = inf;
				y_cur = p1.y + dy;
			}
			if (flat_z)
			{
				inv_z = inf;
				z_cur = p1.z + dz;
			}
		}

		nx = g.nx;
		ny = g.ny;
		nz = g.nz;
		nxy = nx * ny;
		fdx = static_cast<float>(dir_x) * dx;
		fdy = static_cast<float>(dir_y) * dy;
		fdz = static_cast<float>(dir_z) * dz;
		// Every segment moves the voxel along at least one axis, always the
		// same way, so the walk leaves the grid after at most nx+ny+nz
		// segments; the step cap bounds the zero-length steps in between.
		maxSteps = 2 * (nx + ny + nz) + 16;
		if constexpr (TOF)
		{
			// TOF kernel centre along the LOR (mm from p1), loop invariant.
			pc = tofCenter(d_norm, tofValue);
			sigma = tp.sigma;
			norm = tp.norm;
			const float inv_sigma = 1.0f / tp.sigma;
			constexpr float kHalfLog2e = 0.84932180028801904f;  // sqrt(log2(e) / 2)
			hs = 0.5f * d_norm * inv_sigma * kHalfLog2e;
			pcs = pc * inv_sigma * kHalfLog2e;
			dnn = d_norm * tp.norm;
		}

		// First non-empty segment.
		step = 0;
		sx = sy = sz = false;
		bool found = false;
		for (; step < maxSteps && a_cur < amax; step++)
		{
			advance();
			if (a_cur < a_next)
			{
				found = true;
				break;
			}
		}
		if (!found)
			return false;
		step++;
		if constexpr (COMP)
		{
			// Entry voxel from the walk's own plane bookkeeping: the first
			// segment lies just before the next plane of each axis (the plane
			// at a_next for the axes stepped last), so the voxel and the
			// planes the walk steps by can never disagree.  A voxel taken from
			// the segment's midpoint instead is off by one for the whole walk
			// when the first segment is tiny (a TOF window or a piece that
			// starts right before a plane) and the midpoint rounds across that
			// plane.  With the first plane chosen in FP64, a ray within float
			// rounding of a plane (e.g. an LOR between opposite crystals on an
			// image axis) is placed on the side the exact geometry gives.  An
			// axis the ray runs parallel to takes its voxel from the
			// (constant) coordinate in FP64.
			auto fromPlanes = [](bool flat, bool stepped, float cur, float fd,
			                     float q0, float d, int dir, float q1a, int& v)
			{
				if (flat)
				{
					v = static_cast<int>(floor((double(q1a) - double(q0)) * (1.0 / double(d))));
					return;
				}
				const float pre = stepped ? cur - fd : cur;
				const int ip = static_cast<int>(rintf((pre - q0) / d));
				v = dir > 0 ? ip - 1 : ip;
			};
			fromPlanes(flat_x, sx, x_cur, fdx, x0, dx, dir_x, p1.x, vx);
			fromPlanes(flat_y, sy, y_cur, fdy, y0, dy, dir_y, p1.y, vy);
			fromPlanes(flat_z, sz, z_cur, fdz, z0, dz, dir_z, p1.z, vz);
		}
		else
		{
			const float a_mid = 0.5f * (a_cur + a_next);
			vx = static_cast<int>((p1.x + a_mid * (p2.x - p1.x) + g.lx / 2.0f) * inv_dx);
			vy = static_cast<int>((p1.y + a_mid * (p2.y - p1.y) + g.ly / 2.0f) * inv_dy);
			vz = static_cast<int>((p1.z + a_mid * (p2.z - p1.z) + g.lz / 2.0f) * inv_dz);
		}
		if (vx < 0 || vx >= nx || vy < 0 || vy >= ny || vz < 0 || vz >= nz)
			return false;
		if constexpr (COMP)
		{
			// Linear voxel index moved by a per-step delta.  The walk ends at
			// the grid exit (amax); only a rounding-sized last segment can
			// step past a face, and the index check keeps every access inside
			// the image (such a segment adds a weight of ~1e-4 mm to a
			// neighbouring voxel where the mirror walk stops).
			dny = dir_y * nx;
			dnz = dir_z * nxy;
			nvox = static_cast<unsigned>(nxy * nz);
			if constexpr (TILE)
			{
				// x: +1 from even, +3 from odd (into the next 2-wide half or
				// tile); -1 from odd, -3 from even.  y: +2 inside a tile
				// row, 2 nx - 2 into the next; mirrored backwards.
				lin = tileOffset(vx, vy, vz, nx, nxy);
				px = vx & 1;
				py = vy & 1;
				dxo = dir_x > 0 ? 3 : -1;
				dxe = dir_x > 0 ? 1 : -3;
				dyo = dir_y > 0 ? 2 * nx - 2 : -2;
				dye = dir_y > 0 ? 2 : -(2 * nx - 2);
				stepDelta();
			}
			else
			{
				lin = vz * nxy + vy * nx + vx;
				dprev = (sx ? dir_x : 0) + (sy ? dny : 0) + (sz ? dnz : 0);
			}
		}
		else
		{
			off = vz * nxy + vy * nx;
			dir_prev = (sx ? 1 : 0) | (sy ? 2 : 0) | (sz ? 4 : 0);
		}
		return true;
	}

	// Visits the first segment (after a successful begin).
	// TILE, COMP: the offset delta of the axes stepped at the end of this
	// segment, from the current voxel's parities, which then flip.
	__device__ __forceinline__ void stepDelta()
	{
		dprev = (sx ? (px ? dxo : dxe) : 0) + (sy ? (py ? dyo : dye) : 0) + (sz ? dnz : 0);
		px ^= static_cast<int>(sx);
		py ^= static_cast<int>(sy);
	}

	// Offset of the mirror walk's voxel.
	__device__ __forceinline__ int mirrorOffset() const
	{
		if constexpr (TILE)
			return tileOffset(vx, vy, vz, nx, nxy);
		else
			return vx + off;
	}

	template <typename Visit>
	__device__ __forceinline__ void emitFirst(Visit& visit)
	{
		if constexpr (COMP)
			emit(lin, visit);
		else
			emit(mirrorOffset(), visit);
	}

	// One step of the walk: the next crossing, its voxel and its visit;
	// false when the walk has ended.
	template <typename Visit>
	__device__ __forceinline__ bool next(Visit& visit)
	{
		if (!(a_cur < amax))
			return false;
		advance();
		if (a_cur >= a_next)
			return ++step < maxSteps;
		if constexpr (COMP)
		{
			// Following segments: move the voxel along the axes stepped last
			// time.
			lin += dprev;
			if (static_cast<unsigned>(lin) >= nvox)
				return false;
			if constexpr (TILE)
				stepDelta();
			else
				dprev = (sx ? dir_x : 0) + (sy ? dny : 0) + (sz ? dnz : 0);
			emit(lin, visit);
		}
		else
		{
			const int mx = dir_prev & 1, my = (dir_prev >> 1) & 1, mz = (dir_prev >> 2) & 1;
			vx += mx * dir_x;
			vy += my * dir_y;
			vz += mz * dir_z;
			off += my * dir_y * nx + mz * dir_z * nxy;
			if (static_cast<unsigned>(vx) >= static_cast<unsigned>(nx) ||
			    static_cast<unsigned>(vy) >= static_cast<unsigned>(ny) ||
			    static_cast<unsigned>(vz) >= static_cast<unsigned>(nz))
				return false;
			dir_prev = (sx ? 1 : 0) | (sy ? 2 : 0) | (sz ? 4 : 0);
			emit(mirrorOffset(), visit);
		}
		return true;
	}
};

template <bool TOF, bool COMP, bool TILE = false, typename Visit>
__device__ __forceinline__ void siddonWalk(const Geom& g, const float3 p1,
                                           const float3 p2, const TofP& tp,
                                           float tofValue, Visit& visit,
                                           float wlo = 0.f, float whi = 1.f,
                                           int part = 0, int parts = 1)
{
	SiddonWalker<TOF, COMP, TILE> w;
	if (!w.begin(g, p1, p2, tp, tofValue, wlo, whi, part, parts))
		return;
	w.emitFirst(visit);
	while (w.next(visit))
	{
	}
}

// The same walk for the 32 rays of a warp in lock step: every lane takes one
// step per round and the rounds continue while any lane's ray has steps
// left.  The lanes of a warp whose rays step along different axes otherwise
// drift into separate groups that each run the loop with a part of the warp
// (measured on the attenuation walks: 16.5 of 32 threads per instruction).
// Every lane of the warp must call it (alive = false for a lane without a
// ray); each lane's walk is the one siddonWalk makes, step for step.
template <bool TOF, bool COMP, typename Visit>
__device__ __forceinline__ void siddonWalkWarp(bool alive, const Geom& g,
                                               const float3 p1, const float3 p2,
                                               const TofP& tp, float tofValue,
                                               Visit& visit, float wlo = 0.f,
                                               float whi = 1.f)
{
	SiddonWalker<TOF, COMP> w;
	if (alive)
		alive = w.begin(g, p1, p2, tp, tofValue, wlo, whi, 0, 1);
	if (alive)
		w.emitFirst(visit);
	while (__any_sync(0xffffffffu, alive))
	{
		if (alive)
			alive = w.next(visit);
	}
}

// siddonWalkWarp in batches of B crossings: each round every lane takes up
// to B steps, recording the crossings' voxels and weights (o[k] = -1 for a
// step without a crossing or after the walk's end), then hands the batch to
// consume(o, w), which can issue all B image reads before it uses the first
// one.  The crossings reach consume in walk order.
template <bool TOF, bool COMP, int B, typename Consume>
__device__ __forceinline__ void siddonWalkWarpBatched(bool alive, const Geom& g,
                                                      const float3 p1, const float3 p2,
                                                      const TofP& tp, float tofValue,
                                                      Consume& consume, float wlo = 0.f,
                                                      float whi = 1.f)
{
	SiddonWalker<TOF, COMP> w;
	if (alive)
		alive = w.begin(g, p1, p2, tp, tofValue, wlo, whi, 0, 1);
	bool first = alive;
	while (__any_sync(0xffffffffu, alive))
	{
		int o[B];
		float wt[B];
#pragma unroll
		for (int k = 0; k < B; k++)
		{
			o[k] = -1;
			wt[k] = 0.f;
			auto put = [&](int oo, float ww)
			{
				o[k] = oo;
				wt[k] = ww;
			};
			if (k == 0 && first)
			{
				w.emitFirst(put);
				first = false;
			}
			else if (alive)
			{
				alive = w.next(put);
			}
		}
		consume(o, wt);
	}
}

// Number of voxel crossings of the single-ray Siddon walk, estimated in O(1):
// one plus the planes of each axis inside the ray's window (FOV cylinder,
// image slabs, TOF window).  Ties (planes crossed together) count once per
// axis here and once in the walk, so the estimate can exceed the walk's
// count by the number of ties.  Used to group rays of similar length.
template <bool TOF>
__device__ __forceinline__ unsigned crossingEstimate(const Geom& g, float3 p1,
                                                     float3 p2, const TofP& tp,
                                                     float tofValue)
{
	const float ddx = p2.x - p1.x, ddy = p2.y - p1.y, ddz = p2.z - p1.z;
	const float A = ddx * ddx + ddy * ddy;
	float t0 = 0.f, t1 = 1.f;
	if (A != 0.f)
	{
		const float B = 2.0f * (ddx * p1.x + ddy * p1.y);
		const float C = p1.x * p1.x + p1.y * p1.y - g.fovRadius * g.fovRadius;
		const float D = B * B - 4.0f * A * C;
		if (D <= 0.f)
			return 0u;
		const float sq = sqrtf(D);
		t0 = (-B - sq) / (2.0f * A);
		t1 = (-B + sq) / (2.0f * A);
	}
	float amin = fmaxf(0.f, t0), amax = fminf(1.f, t1);
	auto slab = [&](float p, float d, float half)
	{
		if (d != 0.f)
		{
			const float inv = 1.0f / d;
			const float a0 = (-half - p) * inv, a1 = (half - p) * inv;
			amin = fmaxf(amin, fminf(a0, a1));
			amax = fminf(amax, fmaxf(a0, a1));
		}
		else if (p < -half || p > half)
		{
			amax = -1.f;
		}
	};
	slab(p1.x, ddx, 0.5f * g.lx);
	slab(p1.y, ddy, 0.5f * g.ly);
	slab(p1.z, ddz, 0.5f * g.lz);
	if constexpr (TOF)
	{
		float a0, a1;
		tofAlphaRange(tp, sqrtf(A + ddz * ddz), tofValue, a0, a1);
		amin = fmaxf(amin, a0);
		amax = fminf(amax, a1);
	}
	if (!(amin < amax))
		return 0u;
	auto planes = [&](float p, float d, float q0, float dq) -> unsigned
	{
		if (d == 0.f)
			return 0u;
		const float u = floorf((p + amin * d - q0) / dq);
		const float v = floorf((p + amax * d - q0) / dq);
		return static_cast<unsigned>(fabsf(v - u));
	};
	return 1u + planes(p1.x, ddx, -0.5f * g.lx, g.vx) +
	       planes(p1.y, ddy, -0.5f * g.ly, g.vy) + planes(p1.z, ddz, -0.5f * g.lz, g.vz);
}

// Parametric window of the ray p1 -> p2 inside the box of voxels
// [b[0], b[3]] x [b[1], b[4]] x [b[2], b[5]] (inclusive) of grid g; an empty
// box or a miss gives wlo > whi.
__device__ __forceinline__ void boxWindow(const Geom& g, const int* b,
                                          float3 p1, float3 p2, float& wlo,
                                          float& whi)
{
	wlo = 0.f;
	whi = 1.f;
	if (b[3] < b[0])
	{
		wlo = 1.f;
		whi = 0.f;
		return;
	}
	const float lo[3] = {-0.5f * g.lx + b[0] * g.vx, -0.5f * g.ly + b[1] * g.vy,
	                     -0.5f * g.lz + b[2] * g.vz};
	const float hi[3] = {-0.5f * g.lx + (b[3] + 1) * g.vx,
	                     -0.5f * g.ly + (b[4] + 1) * g.vy,
	                     -0.5f * g.lz + (b[5] + 1) * g.vz};
	const float a[3] = {p1.x, p1.y, p1.z};
	const float c[3] = {p2.x, p2.y, p2.z};
#pragma unroll
	for (int k = 0; k < 3; k++)
	{
		float amn, amx;
		const float inv = (a[k] == c[k]) ? 0.f : 1.0f / (c[k] - a[k]);
		slabAlpha<float>(lo[k], hi[k], a[k], c[k], inv, amn, amx);
		wlo = fmaxf(wlo, amn);
		whi = fminf(whi, amx);
	}
}

// ----------------------------------------------------------- multi-ray ----
// Random offsets of the extra rays, as the reference device path draws them:
// curand XORWOW seeded with 13, subsequence = event index in the batch, four
// uniforms per extra ray (i1, j1, i2, j2), each shifted by -0.5.
struct MultiRay
{
	curandState state;
	float3 t1, t2;
	__device__ __forceinline__ void init(unsigned long long id, float3 n1,
	                                     float3 n2)
	{
		curand_init(13ULL, id, 0ULL, &state);
		setDirs(n1, n2);
	}
	// Transverse offset directions of both crystals (without the generator,
	// for offsets read from a table).
	__device__ __forceinline__ void setDirs(float3 n1, float3 n2)
	{
		// cross(n, z) normalised with norm3df, as the reference device code.
		t1 = make_float3(n1.y * 1.f - n1.z * 0.f, n1.z * 0.f - n1.x * 1.f,
		                 n1.x * 0.f - n1.y * 0.f);
		t2 = make_float3(n2.y * 1.f - n2.z * 0.f, n2.z * 0.f - n2.x * 1.f,
		                 n2.x * 0.f - n2.y * 0.f);
		const float l1 = norm3df(t1.x, t1.y, t1.z);
		const float l2 = norm3df(t2.x, t2.y, t2.z);
		t1 = make_float3(t1.x / l1, t1.y / l1, t1.z / l1);
		t2 = make_float3(t2.x / l2, t2.y / l2, t2.z / l2);
	}
	__device__ __forceinline__ void next(float u[4])
	{
		u[0] = curand_uniform(&state) - 0.5f;
		u[1] = curand_uniform(&state) - 0.5f;
		u[2] = curand_uniform(&state) - 0.5f;
		u[3] = curand_uniform(&state) - 0.5f;
	}
	__device__ __forceinline__ void offset(const float u[4], float csz,
	                                       float cst, float3& p1, float3& p2) const
	{
		const float zi1 = u[0] * csz, tj1 = u[1] * cst;
		const float zi2 = u[2] * csz, tj2 = u[3] * cst;
		p1 = make_float3(p1.x + 0.f * zi1 + t1.x * tj1, p1.y + 0.f * zi1 + t1.y * tj1,
		                 p1.z + 1.f * zi1 + t1.z * tj1);
		p2 = make_float3(p2.x + 0.f * zi2 - t2.x * tj2, p2.y + 0.f * zi2 - t2.y * tj2,
		                 p2.z + 1.f * zi2 - t2.z * tj2);
	}
};

// ---------------------------------------------------------------- DD -----
// Integral of the linearly interpolated kernel over [x0, x1]: partial bins at
// both ends plus the whole bins between them, summed bin by bin in the
// reference's order, or (prefix given) as a difference of the row's prefix
// sums, one subtraction instead of a loop over the taps.
__device__ __forceinline__ float psfIntegral(const float* kernel,
                                             int kernelSize, float kernelStep,
                                             float x0, float x1,
                                             const float* prefix = nullptr,
                                             float invStep = 0.f)
{
	const int halfSize = (kernelSize - 1) / 2;
	if (x0 > (halfSize + 1) * kernelStep || x1 < -(halfSize + 1) * kernelStep ||
	    x0 >= x1)
		return 0.f;
	// The prefix form (compensated precision) scales by the reciprocal of the
	// step; the bin-by-bin form divides as the reference does.
	const float x0_s = prefix ? x0 * invStep : x0 / kernelStep;
	const int x0_i = static_cast<int>(floorf(x0_s + halfSize));
	const float tau_0 = x0_s + -(-halfSize + x0_i);
	const float v0_lo = (x0_i < 0 || x0_i >= kernelSize) ? 0.f : __ldg(kernel + x0_i);
	const float v0_hi = (x0_i < -1 || x0_i >= kernelSize - 1) ? 0.f : __ldg(kernel + x0_i + 1);
	const float v0 = v0_lo * (1 - tau_0) + v0_hi * tau_0;
	const float x1_s = prefix ? x1 * invStep : x1 / kernelStep;
	const int x1_i = static_cast<int>(floorf(x1_s + halfSize));
	const float tau_1 = x1_s - (-halfSize + x1_i);
	const float v1_lo = (x1_i < 0 || x1_i >= kernelSize) ? 0.f : __ldg(kernel + x1_i);
	const float v1_hi = (x1_i < -1 || x1_i >= kernelSize - 1) ? 0.f : __ldg(kernel + x1_i + 1);
	const float v1 = v1_lo * (1 - tau_1) + v1_hi * tau_1;
	float out = 0.f;
	if (x0_i == x1_i)
	{
		out = 0.5f * (v0 + v1) * (x1 - x0);
	}
	else
	{
		out += 0.5f * (v0 + v0_hi) * kernelStep * (1 - tau_0);
		out += 0.5f * (v1_lo + v1) * kernelStep * tau_1;
		// Bins entirely outside [-1, kernelSize] contribute exactly zero.
		const int xi_lo = max(x0_i + 1, -1);
		const int xi_hi = min(x1_i, kernelSize + 1);
		if (prefix != nullptr)
		{
			if (xi_hi > xi_lo)
				out += __ldg(prefix + xi_hi + 1) - __ldg(prefix + xi_lo + 1);
		}
		else
		{
			for (int xi = xi_lo; xi < xi_hi; xi++)
			{
				const float v_lo = (xi < 0 || xi >= kernelSize) ? 0.f : __ldg(kernel + xi);
				const float v_hi = (xi + 1 < 0 || xi + 1 >= kernelSize) ? 0.f : __ldg(kernel + xi + 1);
				out += kernelStep * 0.5f * (v_lo + v_hi);
			}
		}
	}
	return out;
}

// Distance-driven footprint of one LOR.  d1, d2: crystal centres relative to
// the image centre; n1, n2: crystal orientations.  visit(offset, weight).
// FASTPSF: PSF integrals from the prefix sums (compensated precision).
// FAST (compensated precision): every division by a value that is constant
// along the LOR or along a row becomes a product with its reciprocal, taken
// once (at most 1 ulp more rounding per weight); otherwise the reference's
// divisions in its order.
template <bool TOF, bool PSF, bool FASTPSF, bool FAST = false, typename Visit>
__device__ __forceinline__ void ddWalk(const Geom& g, const float3 d1,
                                       const float3 d2, const float3 n1,
                                       const float3 n2, float thickness_trans,
                                       float thickness_z, const TofP& tp,
                                       float tofValue, const Psf& psf,
                                       bool forward, Visit& visit,
                                       int part = 0, int parts = 1)
{
	const float3 d12 = f3sub(d1, d2);
	const bool flag_y = fabsf(d12.y) > fabsf(d12.x);
	const float d_norm = sqrtf(d12.x * d12.x + d12.y * d12.y + d12.z * d12.z);
	const float* kern = nullptr;
	const float* kpre = nullptr;
	float ext = 0.f;
	if constexpr (PSF)
	{
		float npx = d2.y - d1.y;
		float npy = d1.x - d2.x;
		const float nn = sqrtf(npx * npx + npy * npy);
		int s_idx = 0;
		if (nn != 0.f)
		{
			npx /= nn;
			npy /= nn;
			const float s = fabsf(d1.x * npx + d1.y * npy);
			const float si = floorf(s / psf.sStep);
			s_idx = (si >= static_cast<float>(psf.num_s - 1)) ? psf.num_s - 1 :
			                                                    static_cast<int>(si);
		}
		kern = (forward ? psf.taps : psf.flipped) + s_idx * psf.size;
		if constexpr (FASTPSF)
			kpre = (forward ? psf.prefix : psf.prefixFlipped) + s_idx * (psf.size + 3);
		ext = static_cast<float>((psf.size + 1) / 2) * psf.kSpacing;
	}
	const float dx = g.vx, dy = g.vy, dz = g.vz;
	const float inv_x = (d1.x == d2.x) ? 0.0f : 1.0f / (d2.x - d1.x);
	const float inv_y = (d1.y == d2.y) ? 0.0f : 1.0f / (d2.y - d1.y);
	const float inv_z = (d1.z == d2.z) ? 0.0f : 1.0f / (d2.z - d1.z);
	float ax_min, ax_max, ay_min, ay_max, az_min, az_max;
	slabAlpha<float>(-0.5f * (g.lx - dx), 0.5f * (g.lx - dx), d1.x, d2.x, inv_x, ax_min, ax_max);
	slabAlpha<float>(-0.5f * (g.ly - dy), 0.5f * (g.ly - dy), d1.y, d2.y, inv_y, ay_min, ay_max);
	slabAlpha<float>(-0.5f * (g.lz - dz), 0.5f * (g.lz - dz), d1.z, d2.z, inv_z, az_min, az_max);
	float amin = fmaxf(fmaxf(fmaxf(0.0f, ax_min), ay_min), az_min);
	float amax = fminf(fminf(fminf(1.0f, ax_max), ay_max), az_max);
	if constexpr (TOF)
	{
		float a0, a1;
		tofAlphaRange(tp, d_norm, tofValue, a0, a1);
		amin = fmaxf(amin, a0);
		amax = fminf(amax, a1);
	}
	const float x_0 = d1.x + amin * (d2.x - d1.x);
	const float y_0 = d1.y + amin * (d2.y - d1.y);
	const float x_1 = d1.x + amax * (d2.x - d1.x);
	const float y_1 = d1.y + amax * (d2.y - d1.y);
	const int x_i_0 = static_cast<int>(floorf(x_0 / dx + 0.5f * (g.nx - 1) + 0.5f));
	const int y_i_0 = static_cast<int>(floorf(y_0 / dy + 0.5f * (g.ny - 1) + 0.5f));
	const int x_i_1 = static_cast<int>(floorf(x_1 / dx + 0.5f * (g.nx - 1) + 0.5f));
	const int y_i_1 = static_cast<int>(floorf(y_1 / dy + 0.5f * (g.ny - 1) + 0.5f));
	const float d1_i = flag_y ? d1.y : d1.x;
	const float d2_i = flag_y ? d2.y : d2.x;
	const float n1_i = flag_y ? n1.y : n1.x;
	const float n2_i = flag_y ? n2.y : n2.x;
	const float n1_xy_norm2 = n1.x * n1.x + n1.y * n1.y;
	const float n1_xy_norm = sqrtf(n1_xy_norm2);
	const float n1_p_x = n1.y / n1_xy_norm;
	const float n1_p_y = -n1.x / n1_xy_norm;
	const float n1_z_norm = sqrtf((n1.x * n1.z) * (n1.x * n1.z) + (n1.y * n1.z) * (n1.y * n1.z) + n1_xy_norm2);
	const float n1_p_i = (n1_i * n1.z) / n1_z_norm;
	const float n1_p_z = -n1_xy_norm2 / n1_z_norm;
	const float n2_xy_norm2 = n2.x * n2.x + n2.y * n2.y;
	const float n2_xy_norm = sqrtf(n2_xy_norm2);
	const float n2_p_x = n2.y / n2_xy_norm;
	const float n2_p_y = -n2.x / n2_xy_norm;
	const float n2_z_norm = sqrtf((n2.x * n2.z) * (n2.x * n2.z) + (n2.y * n2.z) * (n2.y * n2.z) + n2_xy_norm2);
	const float n2_p_i = (n2_i * n2.z) / n2_z_norm;
	const float n2_p_z = -n2_xy_norm2 / n2_z_norm;
	const float htt = thickness_trans * 0.5f;
	const float d1_xy_lo_x = d1.x - htt * n1_p_x, d1_xy_lo_y = d1.y - htt * n1_p_y;
	const float d1_xy_hi_x = d1.x + htt * n1_p_x, d1_xy_hi_y = d1.y + htt * n1_p_y;
	const float d2_xy_lo_x = d2.x - htt * n2_p_x, d2_xy_lo_y = d2.y - htt * n2_p_y;
	const float d2_xy_hi_x = d2.x + htt * n2_p_x, d2_xy_hi_y = d2.y + htt * n2_p_y;
	const float htz = thickness_z * 0.5f;
	const float d1_z_lo_i = d1_i - htz * n1_p_i, d1_z_lo_z = d1.z - htz * n1_p_z;
	const float d1_z_hi_i = d1_i + htz * n1_p_i, d1_z_hi_z = d1.z + htz * n1_p_z;
	const float d2_z_lo_i = d2_i - htz * n2_p_i, d2_z_lo_z = d2.z - htz * n2_p_z;
	const float d2_z_hi_i = d2_i + htz * n2_p_i, d2_z_hi_z = d2.z + htz * n2_p_z;

	int xy_i_0, xy_i_1, nyx;
	float lxy, lyx, dxy, dyx;
	float d1_xy_lo, d1_xy_hi, d2_xy_lo, d2_xy_hi, d1_yx_lo, d1_yx_hi, d2_yx_lo, d2_yx_hi;
	if (flag_y)
	{
		xy_i_0 = max(0, min(y_i_0, y_i_1));
		xy_i_1 = min(g.ny - 1, max(y_i_0, y_i_1));
		lxy = g.ly; dxy = g.vy; lyx = g.lx; dyx = g.vx; nyx = g.nx;
		d1_xy_lo = d1_xy_lo_y; d1_xy_hi = d1_xy_hi_y; d2_xy_lo = d2_xy_lo_y; d2_xy_hi = d2_xy_hi_y;
		d1_yx_lo = d1_xy_lo_x; d1_yx_hi = d1_xy_hi_x; d2_yx_lo = d2_xy_lo_x; d2_yx_hi = d2_xy_hi_x;
	}
	else
	{
		xy_i_0 = max(0, min(x_i_0, x_i_1));
		xy_i_1 = min(g.nx - 1, max(x_i_0, x_i_1));
		lxy = g.lx; dxy = g.vx; lyx = g.ly; dyx = g.vy; nyx = g.ny;
		d1_xy_lo = d1_xy_lo_x; d1_xy_hi = d1_xy_hi_x; d2_xy_lo = d2_xy_lo_x; d2_xy_hi = d2_xy_hi_x;
		d1_yx_lo = d1_xy_lo_y; d1_yx_hi = d1_xy_hi_y; d2_yx_lo = d2_xy_lo_y; d2_yx_hi = d2_xy_hi_y;
	}
	const float dxy_cos_theta =
	    (d1_i != d2_i) ? dxy / (fabsf(d1_i - d2_i) / d_norm) : dxy;
	const int nxy = g.nx * g.ny;
	const float yx_off = static_cast<float>(nyx - 1) / 2.f;
	const float inv_dyx = 1.0f / dyx;
	const float z_off = static_cast<float>(g.nz - 1) * 0.5f;
	const float inv_dz = 1.0f / dz;
	const float half_dyx = dyx * 0.5f;
	// FAST: reciprocals of the denominators that are constant along the LOR.
	const float r_xy_lo = FAST ? 1.0f / (d2_xy_hi - d1_xy_lo) : 0.f;
	const float r_xy_hi = FAST ? 1.0f / (d2_xy_lo - d1_xy_hi) : 0.f;
	const float r_z_lo = FAST ? 1.0f / (d2_z_lo_i - d1_z_lo_i) : 0.f;
	const float r_z_hi = FAST ? 1.0f / (d2_z_hi_i - d1_z_hi_i) : 0.f;
	const float r_i = (FAST && TOF) ? 1.0f / (d2_i - d1_i) : 0.f;
	const float r_step = (FAST && PSF) ? 1.0f / psf.kSpacing : 0.f;

	// Piece `part` of `parts` (several threads per LOR): an even share of the
	// main-axis rows, each row computed exactly as by a single thread.
	int row_lo = xy_i_0, row_hi = xy_i_1;
	if (parts > 1 && xy_i_1 >= xy_i_0)
	{
		const int nrows = xy_i_1 - xy_i_0 + 1;
		row_lo = xy_i_0 + (nrows * part) / parts;
		row_hi = xy_i_0 + (nrows * (part + 1)) / parts - 1;
	}
	for (int xyi = row_lo; xyi <= row_hi; xyi++)
	{
		const float pix_xy = -0.5f * lxy + (static_cast<float>(xyi) + 0.5f) * dxy;
		const float a_xy_lo = FAST ? (pix_xy - d1_xy_lo) * r_xy_lo
		                           : (pix_xy - d1_xy_lo) / (d2_xy_hi - d1_xy_lo);
		const float a_xy_hi = FAST ? (pix_xy - d1_xy_hi) * r_xy_hi
		                           : (pix_xy - d1_xy_hi) / (d2_xy_lo - d1_xy_hi);
		const float a_z_lo = FAST ? (pix_xy - d1_z_lo_i) * r_z_lo
		                          : (pix_xy - d1_z_lo_i) / (d2_z_lo_i - d1_z_lo_i);
		const float a_z_hi = FAST ? (pix_xy - d1_z_hi_i) * r_z_hi
		                          : (pix_xy - d1_z_hi_i) / (d2_z_hi_i - d1_z_hi_i);
		float r0 = d1_yx_lo + a_xy_lo * (d2_yx_hi - d1_yx_lo);
		float r1 = d1_yx_hi + a_xy_hi * (d2_yx_lo - d1_yx_hi);
		if (r0 > r1)
		{
			const float t = r0;
			r0 = r1;
			r1 = t;
		}
		const float widthFrac_yx = r1 - r0;
		const float r0_ov = r0, r1_ov = r1;
		r0 -= ext;
		r1 += ext;
		const int i0 = max(0, static_cast<int>(rintf(r0 * inv_dyx + yx_off)));
		const int i1 = min(nyx - 1, static_cast<int>(rintf(r1 * inv_dyx + yx_off)));
		float zr0 = d1_z_lo_z + a_z_lo * (d2_z_lo_z - d1_z_lo_z);
		float zr1 = d1_z_hi_z + a_z_hi * (d2_z_hi_z - d1_z_hi_z);
		if (zr0 > zr1)
		{
			const float t = zr0;
			zr0 = zr1;
			zr1 = t;
		}
		const float widthFrac_z = zr1 - zr0;
		const int zi0 = max(0, static_cast<int>(rintf(zr0 * inv_dz + z_off)));
		const int zi1 = min(g.nz - 1, static_cast<int>(rintf(zr1 * inv_dz + z_off)));
		float tw = 1.f;
		if constexpr (TOF)
		{
			const float a_lo = FAST ? (pix_xy - d1_i - 0.5f * dxy) * r_i
			                        : (pix_xy - d1_i - 0.5f * dxy) / (d2_i - d1_i);
			const float a_hi = FAST ? (pix_xy - d1_i + 0.5f * dxy) * r_i
			                        : (pix_xy - d1_i + 0.5f * dxy) / (d2_i - d1_i);
			tw = tofWeight(tp, d_norm, tofValue, a_lo * d_norm, a_hi * d_norm);
		}
		// FAST: per-row reciprocals of the footprint widths, and the
		// row factor dxy/cos(theta) folded into the transverse weight.
		const float r_wyx = FAST ? 1.0f / widthFrac_yx : 0.f;
		const float r_wz = FAST ? 1.0f / widthFrac_z : 0.f;
		// The z overlaps of the row's footprint are the same for every
		// transverse voxel of the row: up to kDDZ of them are computed once
		// per row (zq[j] = the factor of voxel zi0 + j, zmask its bit when the
		// voxel overlaps); wider footprints take the per-visit loop.  Same
		// values and visit order either way.
		constexpr int kDDZ = 4;
		float zq[kDDZ];
		unsigned zmask = 0u;
		const bool zfit = zi1 - zi0 < kDDZ;
		if (zfit)
		{
#pragma unroll
			for (int j = 0; j < kDDZ; j++)
			{
				const int zi = zi0 + j;
				const float pix_z = -0.5f * g.lz + (static_cast<float>(zi) + 0.5f) * g.vz;
				const float zp0 = pix_z - g.vz * 0.5f, zp1 = pix_z + g.vz * 0.5f;
				const float wz = fminf(zp1, zr1) - fmaxf(zp0, zr0);
				zq[j] = FAST ? wz * r_wz : wz / widthFrac_z;
				if (zi <= zi1 && zr1 >= zp0 && zr0 < zp1)
					zmask |= 1u << j;
			}
		}
		for (int yxi = i0; yxi <= i1; yxi++)
		{
			const float pix_yx = -0.5f * lyx + (static_cast<float>(yxi) + 0.5f) * dyx;
			const float p0 = pix_yx - half_dyx, p1 = pix_yx + half_dyx;
			if (!(r1 >= p0 && r0 < p1))
				continue;
			float wxy;
			if constexpr (PSF)
			{
				const int halfWidth = (psf.size + 1) / 2;
				const float xa = p0 - r1_ov, xb = p1 - r0_ov;
				if (xa > halfWidth * psf.kSpacing || xb < -halfWidth * psf.kSpacing || xa >= xb)
					wxy = 0.f;
				else
					wxy = psfIntegral(kern, psf.size, psf.kSpacing, xa, xb,
					                  FASTPSF ? kpre : nullptr, r_step);
			}
			else
			{
				wxy = fminf(p1, r1_ov) - fmaxf(p0, r0_ov);
			}
			const float wxy_s = FAST ? wxy * r_wyx * dxy_cos_theta : wxy / widthFrac_yx;
			const int oxy = flag_y ? g.nx * xyi + yxi : g.nx * yxi + xyi;
			if (zfit)
			{
#pragma unroll
				for (int j = 0; j < kDDZ; j++)
				{
					if (zmask & (1u << j))
					{
						const int o = (zi0 + j) * nxy + oxy;
						float w = FAST ? wxy_s * zq[j] : wxy_s * zq[j] * dxy_cos_theta;
						if constexpr (TOF)
							w *= tw;
						visit(o, w);
					}
				}
				continue;
			}
			for (int zi = zi0; zi <= zi1; zi++)
			{
				const float pix_z = -0.5f * g.lz + (static_cast<float>(zi) + 0.5f) * g.vz;
				const float zp0 = pix_z - g.vz * 0.5f, zp1 = pix_z + g.vz * 0.5f;
				if (zr1 >= zp0 && zr0 < zp1)
				{
					const float wz = fminf(zp1, zr1) - fmaxf(zp0, zr0);
					const int o = zi * nxy + oxy;
					float w = FAST ? wxy_s * (wz * r_wz)
					               : wxy_s * (wz / widthFrac_z) * dxy_cos_theta;
					if constexpr (TOF)
						w *= tw;
					visit(o, w);
				}
			}
		}
	}
}

}  // namespace yrtb
