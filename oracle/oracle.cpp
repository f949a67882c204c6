// TEST INFRASTRUCTURE — NOT PART OF THE PRODUCT.
//
// CPU restatement of the YRT-PET 2.0.7 projection hot path, used only to check
// results in tests/ and __graft_entry__.smoke() and in bench.py's CPU leg.
// The product (yrt-pet_b200/) never links, loads or calls this file.
//
// Every routine is templated on the arithmetic type T:
//   T = float  : "mirror" mode.  The reference's FP32 operation order is kept
//                expression by expression (no FMA contraction: built with
//                -ffp-contract=off), so results and the voxel index sequence of
//                each ray are bit-identical to the reference CPU projector.
//   T = double : the FP64 oracle.  Same algorithm evaluated in double; the
//                error budgets of the CUDA path are stated against it.
//
// Parity pins: the float instantiation is compared bit-for-bit with the
// reference library built from its own sources (oracle/ref.mk) and with the
// reference's unit-test known answers (tests/test_oracle_pins.py).
//
// Reference sources followed (paths inside the yrt-pet project):
//   DetRegular::generateLUT           src/datastruct/scanner/DetRegular.cpp:113-183
//   Histogram3D ctor/maps             src/datastruct/projection/Histogram3D.cpp:165-450
//   convertToHistogram3D              src/utils/ReconstructionUtils.cpp:659-720
//   util::get_alpha                   include/yrt-pet/operators/ProjectorUtils.hpp:15-41
//   util::calculateIntegral           include/yrt-pet/operators/ProjectorUtils.hpp:43-98
//   TimeOfFlightHelper                include/yrt-pet/operators/TimeOfFlight.hpp:19-85
//   ProjectorSiddon::project_helper   src/operators/ProjectorSiddon.cpp:478-767
//   ProjectorSiddon fwd/bwd (rays)    src/operators/ProjectorSiddon.cpp:239-369
//   MultiRayGenerator::getRandomLine  src/geometry/MultiRayGenerator.cpp:54-114
//   ProjectorDD::dd_project_ref       src/operators/ProjectorDD.cpp:260-578
//   ProjectionPsfManager              src/operators/ProjectionPsfManager.cpp:27-103
//   OSEM_CPU::computeEMUpdateImage    src/recon/OSEM_CPU.cpp:284-393
//   Image::updateEMThreshold*         src/datastruct/image/Image.cpp:651-833
//   Image::applyThreshold             src/datastruct/image/Image.cpp:594-617

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

namespace orc
{

// Constants as the reference declares them (geometry/Constants.hpp).
constexpr double PI = 3.14159265358979;
constexpr double TWOPI = 6.28318530717959;
constexpr double SPEED_OF_LIGHT_MM_PS = 0.299792458;
constexpr double SPEED_OF_LIGHT_MM_PS_FLT = 0.299792458f;

template <typename T>
struct V3
{
	T x, y, z;
};

template <typename T>
inline V3<T> sub(const V3<T>& a, const V3<T>& b)
{
	return {a.x - b.x, a.y - b.y, a.z - b.z};
}

// Vector3DBase::getNorm: sqrt of (x*x + y*y + z*z) in the vector's type.
template <typename T>
inline T norm3(const V3<T>& v)
{
	return std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
}

struct Image
{
	int64_t nx, ny, nz, nt;
	float length_x, length_y, length_z, off_x, off_y, off_z;
};

// ImageParams::setup (src/datastruct/image/ImageParams.cpp:205-218).
template <typename T>
struct Grid
{
	int64_t nx, ny, nz;
	T lx, ly, lz, vx, vy, vz, fovRadius;
	explicit Grid(const Image& im)
	{
		nx = im.nx;
		ny = im.ny;
		nz = im.nz;
		lx = im.length_x;
		ly = im.length_y;
		lz = im.length_z;
		// vx = length / n (computed in float by the reference).
		const float fvx = im.length_x / static_cast<float>(im.nx);
		const float fvy = im.length_y / static_cast<float>(im.ny);
		const float fvz = im.length_z / static_cast<float>(im.nz);
		float fr = std::max(im.length_x / 2.0f, im.length_y / 2.0f);
		fr -= std::max(fvx, fvy) / 1000.0f;
		if constexpr (sizeof(T) == 4)
		{
			vx = fvx;
			vy = fvy;
			vz = fvz;
			fovRadius = fr;
		}
		else
		{
			vx = static_cast<double>(im.length_x) / im.nx;
			vy = static_cast<double>(im.length_y) / im.ny;
			vz = static_cast<double>(im.length_z) / im.nz;
			fovRadius = std::max(lx / 2.0, ly / 2.0) - std::max(vx, vy) / 1000.0;
		}
	}
};

// ---------------------------------------------------------------- TOF ----
template <typename T>
struct Tof
{
	T sigma, trunc, norm;
	Tof(float fwhm_ps, int n_std)
	{
		if constexpr (sizeof(T) == 4)
		{
			// Mixed float/double arithmetic exactly as TimeOfFlight.hpp:20-33.
			const double tof_width_mm = fwhm_ps * SPEED_OF_LIGHT_MM_PS * 0.5;
			sigma = tof_width_mm / (2 * sqrtf(2 * logf(2)));
			trunc = (n_std <= 0) ? -1.f : n_std * sigma;
			norm = 1 / (std::sqrt(2 * PI) * sigma);
		}
		else
		{
			const double w = fwhm_ps * SPEED_OF_LIGHT_MM_PS * 0.5;
			sigma = w / (2.0 * std::sqrt(2.0 * std::log(2.0)));
			trunc = (n_std <= 0) ? -1.0 : n_std * sigma;
			norm = 1.0 / (std::sqrt(2.0 * M_PI) * sigma);
		}
	}
	// TimeOfFlightHelper::getAlphaRange (TimeOfFlight.hpp:53-72).
	void alphaRange(T& amin, T& amax, T lorNorm, float tof_ps) const
	{
		if (trunc <= T(0))
		{
			amin = 0;
			amax = 1;
			return;
		}
		if constexpr (sizeof(T) == 4)
		{
			const float tof_mm = tof_ps * SPEED_OF_LIGHT_MM_PS_FLT * 0.5;
			amin = std::max(0.0, 0.5 + (tof_mm - trunc) / lorNorm);
			amax = std::min(1.0, 0.5 + (tof_mm + trunc) / lorNorm);
		}
		else
		{
			const double tof_mm = tof_ps * SPEED_OF_LIGHT_MM_PS * 0.5;
			amin = std::max(0.0, 0.5 + (tof_mm - trunc) / lorNorm);
			amax = std::min(1.0, 0.5 + (tof_mm + trunc) / lorNorm);
		}
	}
	// TimeOfFlightHelper::getWeight (TimeOfFlight.hpp:74-84): Gaussian
	// evaluated at the segment midpoint (not integrated over the segment).
	T weight(T lorNorm, float tof_ps, T lo, T hi) const
	{
		if constexpr (sizeof(T) == 4)
		{
			const float tof_mm = tof_ps * SPEED_OF_LIGHT_MM_PS_FLT * 0.5;
			const float pc = 0.5 * lorNorm + tof_mm;
			const float xc = (0.5f * (lo + hi) - pc) / sigma;
#ifdef ORC_EXP_DOUBLE
			return static_cast<float>(std::exp(static_cast<double>(-0.5f * xc * xc)) * norm);
#else
			return std::exp(-0.5f * xc * xc) * norm;
#endif
		}
		else
		{
			const double tof_mm = tof_ps * SPEED_OF_LIGHT_MM_PS * 0.5;
			const double pc = 0.5 * lorNorm + tof_mm;
			const double xc = (0.5 * (lo + hi) - pc) / sigma;
			return std::exp(-0.5 * xc * xc) * norm;
		}
	}
};

// util::get_alpha (ProjectorUtils.hpp:15-41).
template <typename T>
inline void getAlpha(T r0, T r1, T p1, T p2, T inv, T& amin, T& amax)
{
	amin = 0.0;
	amax = 1.0;
	if (p1 != p2)
	{
		const T a0 = (r0 - p1) * inv;
		const T a1 = (r1 - p1) * inv;
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
		amax = 0.0;
		amin = 1.0;
	}
}

// ------------------------------------------------------------ Siddon ----
// Visitor receives (flat voxel offset inside a frame, weight).
template <typename T, bool INCR, bool TOF, typename Visit>
void siddon(const Grid<T>& g, V3<T> p1, V3<T> p2, const Tof<T>* tof,
            float tofValue, Visit&& visit)
{
	// 1. Intersection with the centred FOV cylinder (ProjectorSiddon.cpp:495-518).
	T t0, t1;
	const T A = (p2.x - p1.x) * (p2.x - p1.x) + (p2.y - p1.y) * (p2.y - p1.y);
	const T B = T(2) * ((p2.x - p1.x) * p1.x + (p2.y - p1.y) * p1.y);
	const T C = p1.x * p1.x + p1.y * p1.y - g.fovRadius * g.fovRadius;
	const T Delta = B * B - T(4) * A * C;
	if (A != T(0))
	{
		if (Delta <= T(0))
			return;
		// sqrt of a float is the float overload in the reference translation
		// unit (checked bit-for-bit against the compiled reference).
		const T sq = std::sqrt(Delta);
		t0 = static_cast<T>((-B - sq) / (T(2) * A));
		t1 = static_cast<T>((-B + sq) / (T(2) * A));
	}
	else
	{
		t0 = 0;
		t1 = 1;
	}

	const T d_norm = norm3(sub(p1, p2));
	const bool flat_x = (p1.x == p2.x);
	const bool flat_y = (p1.y == p2.y);
	const bool flat_z = (p1.z == p2.z);
	const T inv_x = flat_x ? T(0) : T(1) / (p2.x - p1.x);
	const T inv_y = flat_y ? T(0) : T(1) / (p2.y - p1.y);
	const T inv_z = flat_z ? T(0) : T(1) / (p2.z - p1.z);
	const int64_t dir_x = (inv_x >= T(0)) ? 1 : -1;
	const int64_t dir_y = (inv_y >= T(0)) ? 1 : -1;
	const int64_t dir_z = (inv_z >= T(0)) ? 1 : -1;

	// 2. Intersection with the image volume (:531-560).
	const T dx = g.vx, dy = g.vy, dz = g.vz;
	const T inv_dx = T(1) / dx, inv_dy = T(1) / dy, inv_dz = T(1) / dz;
	const T x0 = -g.lx * T(0.5), x1 = g.lx * T(0.5);
	const T y0 = -g.ly * T(0.5), y1 = g.ly * T(0.5);
	const T z0 = -g.lz * T(0.5), z1 = g.lz * T(0.5);
	T ax_min, ax_max, ay_min, ay_max, az_min, az_max;
	getAlpha<T>(T(-0.5) * g.lx, T(0.5) * g.lx, p1.x, p2.x, inv_x, ax_min, ax_max);
	getAlpha<T>(T(-0.5) * g.ly, T(0.5) * g.ly, p1.y, p2.y, inv_y, ay_min, ay_max);
	getAlpha<T>(T(-0.5) * g.lz, T(0.5) * g.lz, p1.z, p2.z, inv_z, az_min, az_max);
	T amin = std::max({T(0), t0, ax_min, ay_min, az_min});
	T amax = std::min({T(1), t1, ax_max, ay_max, az_max});
	if constexpr (TOF)
	{
		T amin_tof, amax_tof;
		tof->alphaRange(amin_tof, amax_tof, d_norm, tofValue);
		amin = std::max(amin, amin_tof);
		amax = std::min(amax, amax_tof);
	}

	T a_cur = amin;
	T a_next = -1;
	T x_cur = (inv_x > T(0)) ? x0 : x1;
	T y_cur = (inv_y > T(0)) ? y0 : y1;
	T z_cur = (inv_z > T(0)) ? z0 : z1;
	if ((inv_x >= T(0) && p1.x > x1) || (inv_x < T(0) && p1.x < x0) ||
	    (inv_y >= T(0) && p1.y > y1) || (inv_y < T(0) && p1.y < y0) ||
	    (inv_z >= T(0) && p1.z > z1) || (inv_z < T(0) && p1.z < z0))
		return;

	// Move the starting plane inside the FOV (:573-594).
	T ax_next = flat_x ? std::numeric_limits<T>::max() : ax_min;
	if (!flat_x)
	{
		const int64_t kx = static_cast<int64_t>(std::ceil(
		    static_cast<T>(dir_x) * (a_cur * (p2.x - p1.x) - x_cur + p1.x) / dx));
		x_cur += static_cast<T>(kx * dir_x) * dx;
		ax_next = (x_cur - p1.x) * inv_x;
	}
	T ay_next = flat_y ? std::numeric_limits<T>::max() : ay_min;
	if (!flat_y)
	{
		const int64_t ky = static_cast<int64_t>(std::ceil(
		    static_cast<T>(dir_y) * (a_cur * (p2.y - p1.y) - y_cur + p1.y) / dy));
		y_cur += static_cast<T>(ky * dir_y) * dy;
		ay_next = (y_cur - p1.y) * inv_y;
	}
	T az_next = flat_z ? std::numeric_limits<T>::max() : az_min;
	if (!flat_z)
	{
		const int64_t kz = static_cast<int64_t>(std::ceil(
		    static_cast<T>(dir_z) * (a_cur * (p2.z - p1.z) - z_cur + p1.z) / dz));
		z_cur += static_cast<T>(kz * dir_z) * dz;
		az_next = (z_cur - p1.z) * inv_z;
	}

	bool flag_first = true;
	int64_t vx = -1, vy = -1, vz = -1;
	int dir_prev = -1, dir_next = -1;
	const int64_t nx = g.nx, ny = g.ny, nz = g.nz, num_xy = nx * ny;
	int64_t off = 0;
	T axp = ax_next, ayp = ay_next, azp = az_next;

	// 3. Incremental walk (:622-766).
	bool done = false;
	while (a_cur < amax && !done)
	{
		dir_next = 0;
		if (axp <= ayp && axp <= azp)
		{
			a_next = ax_next;
			x_cur += static_cast<T>(dir_x) * dx;
			ax_next = (x_cur - p1.x) * inv_x;
			dir_next |= 1;
		}
		if (ayp <= axp && ayp <= azp)
		{
			a_next = ay_next;
			y_cur += static_cast<T>(dir_y) * dy;
			ay_next = (y_cur - p1.y) * inv_y;
			dir_next |= 2;
		}
		if (azp <= axp && azp <= ayp)
		{
			a_next = az_next;
			z_cur += static_cast<T>(dir_z) * dz;
			az_next = (z_cur - p1.z) * inv_z;
			dir_next |= 4;
		}
		if (a_next > amax)
			a_next = amax;
		if (a_cur >= a_next)
		{
			axp = ax_next;
			ayp = ay_next;
			azp = az_next;
			continue;
		}
		T tof_w = 1;
		const T a_mid = T(0.5) * (a_cur + a_next);
		if constexpr (TOF)
			tof_w = tof->weight(d_norm, tofValue, a_cur * d_norm,
			                    a_next * d_norm);
		if (!INCR || flag_first)
		{
			vx = static_cast<int64_t>((p1.x + a_mid * (p2.x - p1.x) + g.lx / T(2)) * inv_dx);
			vy = static_cast<int64_t>((p1.y + a_mid * (p2.y - p1.y) + g.ly / T(2)) * inv_dy);
			vz = static_cast<int64_t>((p1.z + a_mid * (p2.z - p1.z) + g.lz / T(2)) * inv_dz);
			off = vz * num_xy + vy * nx;
			flag_first = false;
			if (vx < 0 || vx >= nx || vy < 0 || vy >= ny || vz < 0 || vz >= nz)
				done = true;
		}
		else
		{
			if (dir_prev & 1)
			{
				vx += dir_x;
				if (vx < 0 || vx >= nx)
					done = true;
			}
			if (dir_prev & 2)
			{
				vy += dir_y;
				if (vy < 0 || vy >= ny)
					done = true;
				else
					off += dir_y * nx;
			}
			if (dir_prev & 4)
			{
				vz += dir_z;
				if (vz < 0 || vz >= nz)
					done = true;
				else
					off += dir_z * num_xy;
			}
		}
		if (done)
			continue;
		dir_prev = dir_next;
		T w = (a_next - a_cur) * d_norm;
		if constexpr (TOF)
			w *= tof_w;
		visit(vx + off, w);
		a_cur = a_next;
		axp = ax_next;
		ayp = ay_next;
		azp = az_next;
	}
}

template <typename T>
struct Ray
{
	V3<T> p1, p2;
};

// Offsets a LOR for one extra ray (MultiRayGenerator::getRandomLine,
// MultiRayGenerator.cpp:72-114; the same geometry as the device
// moveLineToRandomOffset, SiddonKernels.cuh:45-84).  u = 4 uniforms already
// shifted to [-0.5, 0.5]: (i1, j1, i2, j2).
template <typename T>
Ray<T> offsetRay(const Ray<T>& r, const V3<float>& n1, const V3<float>& n2,
                 const float* u, float csz, float cst)
{
	// cross(n, z) = (n.y, -n.x, 0), normalised.
	auto perp = [](const V3<float>& n)
	{
		float x = n.y, y = -n.x;
		float nn = std::sqrt(x * x + y * y);
		if (nn > 10e-25)
		{
			x /= nn;
			y /= nn;
		}
		return V3<float>{x, y, 0.f};
	};
	const V3<float> t1 = perp(n1), t2 = perp(n2);
	Ray<T> o;
	const float zi1 = u[0] * csz, tj1 = u[1] * cst;
	const float zi2 = u[2] * csz, tj2 = u[3] * cst;
	o.p1 = {static_cast<T>(r.p1.x + T(0) * zi1 + t1.x * tj1),
	        static_cast<T>(r.p1.y + T(0) * zi1 + t1.y * tj1),
	        static_cast<T>(r.p1.z + T(1) * zi1 + t1.z * tj1)};
	o.p2 = {static_cast<T>(r.p2.x + T(0) * zi2 - t2.x * tj2),
	        static_cast<T>(r.p2.y + T(0) * zi2 - t2.y * tj2),
	        static_cast<T>(r.p2.z + T(1) * zi2 - t2.z * tj2)};
	return o;
}

// ---------------------------------------------------------------- DD ----
struct Psf
{
	int num_s = 0, size = 0;
	float sStep = 0, kSpacing = 0;
	const float* taps = nullptr;     // num_s * size
	std::vector<float> flipped;      // adjoint taps
};

// util::calculateIntegral (ProjectorUtils.hpp:43-98).
template <typename T>
T psfIntegral(const float* kernel, int kernelSize, T kernelStep, T x0, T x1)
{
	const int halfSize = (kernelSize - 1) / 2;
	if (x0 > (halfSize + 1) * kernelStep || x1 < -(halfSize + 1) * kernelStep ||
	    x0 >= x1)
		return 0;
	const T x0_s = x0 / kernelStep;
	const int x0_i = static_cast<int>(std::floor(x0_s + halfSize));
	const T tau_0 = x0_s + -(-halfSize + x0_i);
	const T v0_lo = (x0_i < 0 || x0_i >= kernelSize) ? T(0) : T(kernel[x0_i]);
	const T v0_hi = (x0_i < -1 || x0_i >= kernelSize - 1) ? T(0) : T(kernel[x0_i + 1]);
	const T v0 = v0_lo * (1 - tau_0) + v0_hi * tau_0;
	const T x1_s = x1 / kernelStep;
	const int x1_i = static_cast<int>(std::floor(x1_s + halfSize));
	const T tau_1 = x1_s - (-halfSize + x1_i);
	const T v1_lo = (x1_i < 0 || x1_i >= kernelSize) ? T(0) : T(kernel[x1_i]);
	const T v1_hi = (x1_i < -1 || x1_i >= kernelSize - 1) ? T(0) : T(kernel[x1_i + 1]);
	const T v1 = v1_lo * (1 - tau_1) + v1_hi * tau_1;
	T out = 0;
	if (x0_i == x1_i)
	{
		out = T(0.5) * (v0 + v1) * (x1 - x0);
	}
	else
	{
		out += T(0.5) * (v0 + v0_hi) * kernelStep * (1 - tau_0);
		out += T(0.5) * (v1_lo + v1) * kernelStep * tau_1;
		for (int xi = x0_i + 1; xi < x1_i; xi++)
		{
			const T v_lo = (xi < 0 || xi >= kernelSize) ? T(0) : T(kernel[xi]);
			const T v_hi = (xi + 1 < 0 || xi + 1 >= kernelSize) ? T(0) : T(kernel[xi + 1]);
			out += kernelStep * T(0.5) * (v_lo + v_hi);
		}
	}
	return out;
}

// ProjectionPsfManager::getKernel (ProjectionPsfManager.cpp:62-88).
template <typename T>
const float* psfKernel(const Psf& psf, const V3<T>& p1, const V3<T>& p2,
                       bool flipped)
{
	float npx = p2.y - p1.y;
	float npy = p1.x - p2.x;
	const float nn = std::sqrt(npx * npx + npy * npy);
	size_t s_idx = 0;
	if (nn != 0)
	{
		npx /= nn;
		npy /= nn;
		const float s = std::abs(static_cast<float>(p1.x) * npx + static_cast<float>(p1.y) * npy);
		s_idx = std::min(static_cast<size_t>(std::floor(s / psf.sStep)),
		                 static_cast<size_t>(psf.num_s - 1));
	}
	return flipped ? psf.flipped.data() + s_idx * psf.size :
	                 psf.taps + s_idx * psf.size;
}

// ProjectorDD::getOverlap_safe with and without PSF (ProjectorDD.cpp:234-255).
template <typename T>
inline T ddOverlap(T p0, T p1, T d0, T d1, const Psf* psf, const float* kern)
{
	if (psf)
	{
		const int halfWidth = (psf->size + 1) / 2;
		const T x0 = p0 - d1, x1 = p1 - d0;
		if (x0 > halfWidth * T(psf->kSpacing) || x1 < -halfWidth * T(psf->kSpacing) || x0 >= x1)
			return 0;
		return psfIntegral<T>(kern, psf->size, T(psf->kSpacing), x0, x1);
	}
	return std::min(p1, d1) - std::max(p0, d0);
}

template <typename T, typename Visit>
void dd(const Grid<T>& g, V3<T> d1, V3<T> d2, V3<T> n1, V3<T> n2,
        float thickness_trans, float thickness_z, const Tof<T>* tof,
        float tofValue, const Psf* psf, bool forward, Visit&& visit)
{
	const V3<T> d12 = sub(d1, d2);
	const bool flag_y = std::abs(d12.y) > std::abs(d12.x);
	const T d_norm = norm3(d12);
	const float* kern = nullptr;
	T ext = 0;
	if (psf)
	{
		kern = psfKernel<T>(*psf, d1, d2, !forward);
		ext = static_cast<T>((psf->size + 1) / 2 * psf->kSpacing);
	}
	const int64_t num_xy = g.nx * g.ny;
	const T dx = g.vx, dy = g.vy, dz = g.vz;
	const T inv_x = (d1.x == d2.x) ? T(0) : T(1) / (d2.x - d1.x);
	const T inv_y = (d1.y == d2.y) ? T(0) : T(1) / (d2.y - d1.y);
	const T inv_z = (d1.z == d2.z) ? T(0) : T(1) / (d2.z - d1.z);
	T ax_min, ax_max, ay_min, ay_max, az_min, az_max;
	getAlpha<T>(T(-0.5) * (g.lx - dx), T(0.5) * (g.lx - dx), d1.x, d2.x, inv_x, ax_min, ax_max);
	getAlpha<T>(T(-0.5) * (g.ly - dy), T(0.5) * (g.ly - dy), d1.y, d2.y, inv_y, ay_min, ay_max);
	getAlpha<T>(T(-0.5) * (g.lz - dz), T(0.5) * (g.lz - dz), d1.z, d2.z, inv_z, az_min, az_max);
	T amin = std::max({T(0), ax_min, ay_min, az_min});
	T amax = std::min({T(1), ax_max, ay_max, az_max});
	if (tof)
	{
		T a0, a1;
		tof->alphaRange(a0, a1, d_norm, tofValue);
		amin = std::max(amin, a0);
		amax = std::min(amax, a1);
	}
	const T x_0 = d1.x + amin * (d2.x - d1.x);
	const T y_0 = d1.y + amin * (d2.y - d1.y);
	const T x_1 = d1.x + amax * (d2.x - d1.x);
	const T y_1 = d1.y + amax * (d2.y - d1.y);
	const int64_t x_i_0 = static_cast<int64_t>(std::floor(x_0 / dx + T(0.5) * (g.nx - 1) + T(0.5)));
	const int64_t y_i_0 = static_cast<int64_t>(std::floor(y_0 / dy + T(0.5) * (g.ny - 1) + T(0.5)));
	const int64_t x_i_1 = static_cast<int64_t>(std::floor(x_1 / dx + T(0.5) * (g.nx - 1) + T(0.5)));
	const int64_t y_i_1 = static_cast<int64_t>(std::floor(y_1 / dy + T(0.5) * (g.ny - 1) + T(0.5)));
	T d1_i, d2_i, n1_i, n2_i;
	if (flag_y)
	{
		d1_i = d1.y; d2_i = d2.y; n1_i = n1.y; n2_i = n2.y;
	}
	else
	{
		d1_i = d1.x; d2_i = d2.x; n1_i = n1.x; n2_i = n2.x;
	}
	const T n1_xy_norm2 = n1.x * n1.x + n1.y * n1.y;
	const T n1_xy_norm = std::sqrt(n1_xy_norm2);
	const T n1_p_x = n1.y / n1_xy_norm;
	const T n1_p_y = -n1.x / n1_xy_norm;
	const T n1_z_norm = std::sqrt((n1.x * n1.z) * (n1.x * n1.z) + (n1.y * n1.z) * (n1.y * n1.z) + n1_xy_norm2);
	const T n1_p_i = (n1_i * n1.z) / n1_z_norm;
	const T n1_p_z = -n1_xy_norm2 / n1_z_norm;
	const T n2_xy_norm2 = n2.x * n2.x + n2.y * n2.y;
	const T n2_xy_norm = std::sqrt(n2_xy_norm2);
	const T n2_p_x = n2.y / n2_xy_norm;
	const T n2_p_y = -n2.x / n2_xy_norm;
	const T n2_z_norm = std::sqrt((n2.x * n2.z) * (n2.x * n2.z) + (n2.y * n2.z) * (n2.y * n2.z) + n2_xy_norm2);
	const T n2_p_i = (n2_i * n2.z) / n2_z_norm;
	const T n2_p_z = -n2_xy_norm2 / n2_z_norm;

	const T htt = T(thickness_trans) * T(0.5);
	const T d1_xy_lo_x = d1.x - htt * n1_p_x, d1_xy_lo_y = d1.y - htt * n1_p_y;
	const T d1_xy_hi_x = d1.x + htt * n1_p_x, d1_xy_hi_y = d1.y + htt * n1_p_y;
	const T d2_xy_lo_x = d2.x - htt * n2_p_x, d2_xy_lo_y = d2.y - htt * n2_p_y;
	const T d2_xy_hi_x = d2.x + htt * n2_p_x, d2_xy_hi_y = d2.y + htt * n2_p_y;
	const T htz = T(thickness_z) * T(0.5);
	const T d1_z_lo_i = d1_i - htz * n1_p_i, d1_z_lo_z = d1.z - htz * n1_p_z;
	const T d1_z_hi_i = d1_i + htz * n1_p_i, d1_z_hi_z = d1.z + htz * n1_p_z;
	const T d2_z_lo_i = d2_i - htz * n2_p_i, d2_z_lo_z = d2.z - htz * n2_p_z;
	const T d2_z_hi_i = d2_i + htz * n2_p_i, d2_z_hi_z = d2.z + htz * n2_p_z;

	int64_t xy_i_0, xy_i_1, nyx;
	T lxy, lyx, dxy, dyx;
	T d1_xy_lo, d1_xy_hi, d2_xy_lo, d2_xy_hi, d1_yx_lo, d1_yx_hi, d2_yx_lo, d2_yx_hi;
	if (flag_y)
	{
		xy_i_0 = std::max<int64_t>(0, std::min(y_i_0, y_i_1));
		xy_i_1 = std::min<int64_t>(g.ny - 1, std::max(y_i_0, y_i_1));
		lxy = g.ly; dxy = g.vy; lyx = g.lx; dyx = g.vx; nyx = g.nx;
		d1_xy_lo = d1_xy_lo_y; d1_xy_hi = d1_xy_hi_y; d2_xy_lo = d2_xy_lo_y; d2_xy_hi = d2_xy_hi_y;
		d1_yx_lo = d1_xy_lo_x; d1_yx_hi = d1_xy_hi_x; d2_yx_lo = d2_xy_lo_x; d2_yx_hi = d2_xy_hi_x;
	}
	else
	{
		xy_i_0 = std::max<int64_t>(0, std::min(x_i_0, x_i_1));
		xy_i_1 = std::min<int64_t>(g.nx - 1, std::max(x_i_0, x_i_1));
		lxy = g.lx; dxy = g.vx; lyx = g.ly; dyx = g.vy; nyx = g.ny;
		d1_xy_lo = d1_xy_lo_x; d1_xy_hi = d1_xy_hi_x; d2_xy_lo = d2_xy_lo_x; d2_xy_hi = d2_xy_hi_x;
		d1_yx_lo = d1_xy_lo_y; d1_yx_hi = d1_xy_hi_y; d2_yx_lo = d2_xy_lo_y; d2_yx_hi = d2_xy_hi_y;
	}
	T dxy_cos_theta;
	if (d1_i != d2_i)
		dxy_cos_theta = dxy / (std::abs(d1_i - d2_i) / d_norm);
	else
		dxy_cos_theta = dxy;

	for (int64_t xyi = xy_i_0; xyi <= xy_i_1; xyi++)
	{
		const T pix_xy = T(-0.5) * lxy + (static_cast<T>(xyi) + T(0.5)) * dxy;
		const T a_xy_lo = (pix_xy - d1_xy_lo) / (d2_xy_hi - d1_xy_lo);
		const T a_xy_hi = (pix_xy - d1_xy_hi) / (d2_xy_lo - d1_xy_hi);
		const T a_z_lo = (pix_xy - d1_z_lo_i) / (d2_z_lo_i - d1_z_lo_i);
		const T a_z_hi = (pix_xy - d1_z_hi_i) / (d2_z_hi_i - d1_z_hi_i);
		T r0 = d1_yx_lo + a_xy_lo * (d2_yx_hi - d1_yx_lo);
		T r1 = d1_yx_hi + a_xy_hi * (d2_yx_lo - d1_yx_hi);
		if (r0 > r1)
			std::swap(r0, r1);
		const T widthFrac_yx = r1 - r0;
		const T r0_ov = r0, r1_ov = r1;
		r0 -= ext;
		r1 += ext;
		const T yx_off = (nyx - 1) / T(2);
		const T inv_dyx = T(1) / dyx;
		const int64_t i0 = std::max<int64_t>(0, static_cast<int64_t>(std::rint(r0 * inv_dyx + yx_off)));
		const int64_t i1 = std::min<int64_t>(nyx - 1, static_cast<int64_t>(std::rint(r1 * inv_dyx + yx_off)));
		for (int64_t yxi = i0; yxi <= i1; yxi++)
		{
			const T pix_yx = T(-0.5) * lyx + (static_cast<T>(yxi) + T(0.5)) * dyx;
			T z0 = d1_z_lo_z + a_z_lo * (d2_z_lo_z - d1_z_lo_z);
			T z1 = d1_z_hi_z + a_z_hi * (d2_z_hi_z - d1_z_hi_z);
			if (z0 > z1)
				std::swap(z0, z1);
			const T widthFrac_z = z1 - z0;
			const T half_dyx = dyx * T(0.5);
			const T p0 = pix_yx - half_dyx, p1 = pix_yx + half_dyx;
			if (r1 >= p0 && r0 < p1)
			{
				const T wxy = ddOverlap<T>(p0, p1, r0_ov, r1_ov, psf, kern);
				const T wxy_s = wxy / widthFrac_yx;
				const T z_off = (g.nz - 1) * T(0.5);
				const T inv_dz = T(1) / dz;
				const int64_t zi0 = std::max<int64_t>(0, static_cast<int64_t>(std::rint(z0 * inv_dz + z_off)));
				const int64_t zi1 = std::min<int64_t>(g.nz - 1, static_cast<int64_t>(std::rint(z1 * inv_dz + z_off)));
				for (int64_t zi = zi0; zi <= zi1; zi++)
				{
					const T pix_z = T(-0.5) * g.lz + (static_cast<T>(zi) + T(0.5)) * g.vz;
					T tw = 1;
					if (tof)
					{
						const T a_lo = (pix_xy - d1_i - T(0.5) * dxy) / (d2_i - d1_i);
						const T a_hi = (pix_xy - d1_i + T(0.5) * dxy) / (d2_i - d1_i);
						tw = tof->weight(d_norm, tofValue, a_lo * d_norm, a_hi * d_norm);
					}
					const T zp0 = pix_z - g.vz * T(0.5), zp1 = pix_z + g.vz * T(0.5);
					if (z1 >= zp0 && z0 < zp1)
					{
						const T wz = std::min(zp1, z1) - std::max(zp0, z0);
						const T wz_s = wz / widthFrac_z;
						int64_t o = zi * num_xy;
						if (flag_y)
							o += g.nx * xyi + yxi;
						else
							o += g.nx * yxi + xyi;
						T w = wxy_s * wz_s * dxy_cos_theta;
						if (tof)
							w *= tw;
						visit(o, w);
					}
				}
			}
		}
	}
}

// ------------------------------------------------------ parallel loops ----
template <typename F>
void parallelFor(size_t n, int threads, F&& f)
{
	if (threads <= 1 || n < 256)
	{
		for (size_t i = 0; i < n; i++)
			f(i, 0);
		return;
	}
	std::vector<std::thread> pool;
	std::atomic<size_t> next{0};
	for (int t = 0; t < threads; t++)
		pool.emplace_back(
		    [&, t]
		    {
			    for (;;)
			    {
				    const size_t b = next.fetch_add(4096);
				    if (b >= n)
					    break;
				    const size_t e = std::min(n, b + 4096);
				    for (size_t i = b; i < e; i++)
					    f(i, t);
			    }
		    });
	for (auto& th : pool)
		th.join();
}

}  // namespace orc

using namespace orc;

extern "C" {

struct orc_scanner
{
	float axialFOV, crystalSize_z, crystalSize_trans, crystalDepth,
	    scannerRadius;
	uint64_t detsPerRing, numRings, numDOI, maxRingDiff, minAngDiff,
	    detsPerBlock;
};

// Projection options shared by the Siddon / DD entry points.
struct orc_proj
{
	int projector;         // 0 Siddon, 1 DD
	int incremental;       // Siddon only: 1 = FLAG_INCR walk, 0 = slow walk
	float tof_fwhm_ps;     // <= 0: no TOF
	int tof_n_std;
	int num_rays;          // Siddon multi-ray (needs orients and ray_offsets)
	float crystal_z, crystal_trans;
	int psf_num_s, psf_size;
	float psf_s_step, psf_k_spacing;
	const float* psf_taps;  // psf_num_s * psf_size, nullable
	int threads;
};

// DetRegular::generateLUT in float, as the reference computes it.
int orc_scanner_lut(const orc_scanner* s, float* out)
{
	const size_t numBlocks = s->detsPerRing / s->detsPerBlock;
	const float blockLength = s->crystalSize_trans * s->detsPerBlock;
	for (size_t doi = 0; doi < s->numDOI; doi++)
	{
		const float blockDistance = s->scannerRadius + s->crystalDepth * doi;
		for (size_t ring = 0; ring < s->numRings; ring++)
		{
			const float zGap = s->axialFOV / ((float)s->numRings);
			const float zPos = -s->axialFOV / 2.0 + (ring + 0.5f) * zGap;
			for (size_t block = 0; block < numBlocks; block++)
			{
				const float blockAngle = block * TWOPI / numBlocks;
				const float xBlock = (blockDistance + 0.5f * s->crystalDepth) * std::cos(blockAngle);
				const float yBlock = (blockDistance + 0.5f * s->crystalDepth) * std::sin(blockAngle);
				for (size_t det = 0; det < s->detsPerBlock; det++)
				{
					float rel = 0.0;
					if (s->detsPerBlock != 1)
						rel = -0.5 + (det + 0.5) / (float)s->detsPerBlock;
					const float rx = rel * std::cos(blockAngle + PI / 2.0);
					const float ry = rel * std::sin(blockAngle + PI / 2.0);
					const size_t idx = det + block * s->detsPerBlock +
					                   ring * s->detsPerRing +
					                   doi * (s->numRings * s->detsPerRing);
					out[idx * 6 + 0] = xBlock + blockLength * rx;
					out[idx * 6 + 1] = yBlock + blockLength * ry;
					out[idx * 6 + 2] = zPos;
					out[idx * 6 + 3] = std::cos(blockAngle);
					out[idx * 6 + 4] = std::sin(blockAngle);
					out[idx * 6 + 5] = 0.0f;
				}
			}
		}
	}
	return 0;
}

// ----------------------------------------------------------- Histogram3D --
struct H3
{
	uint64_t numR, numPhi, numZBin, numZBinDiff, rCut, numDOIPoss;
	uint64_t dpr, rings, ndoi, mrd;
	std::vector<int64_t> ringMap;  // dpr*dpr -> r_ring*dpr+phi or -1
	explicit H3(const orc_scanner* s)
	{
		dpr = s->detsPerRing;
		rings = s->numRings;
		ndoi = s->numDOI;
		mrd = s->maxRingDiff;
		rCut = s->minAngDiff / 2;
		if (s->minAngDiff % 2 != 0 && dpr % 4 == 0)
			rCut++;
		numDOIPoss = ndoi * ndoi;
		numR = numDOIPoss * (dpr / 2 + 1 - s->minAngDiff);
		numPhi = dpr;
		uint64_t nz = (mrd + 1) * rings - (mrd * (mrd + 1)) / 2;
		numZBinDiff = nz - rings;
		numZBin = nz + numZBinDiff;
		ringMap.assign(dpr * dpr, -1);
		for (uint64_t phi = 0; phi < numPhi; phi++)
			for (uint64_t r = 0; r < numR / numDOIPoss; r++)
			{
				uint32_t a, b;
				pairInRing(r, phi, a, b);
				ringMap[a * dpr + b] = static_cast<int64_t>(r * dpr + phi);
			}
	}
	// Histogram3D::getDetPairInSameRing (Histogram3D.cpp:428-450).
	void pairInRing(uint64_t r_ring, uint64_t phi, uint32_t& d1, uint32_t& d2) const
	{
		const int n = static_cast<int>(dpr);
		const int r = static_cast<int>(r_ring);
		int d02 = n / 2;
		if (phi % 2 != 0)
			d02 = n / 2 + 1;
		int dr1 = 0 + (r - n / 4 + static_cast<int>(rCut));
		int dr2 = d02 - (r - n / 4 + static_cast<int>(rCut));
		if (dr1 < 0)
			dr1 += n;
		if (dr2 < 0)
			dr2 += n;
		d1 = static_cast<uint32_t>((dr1 + static_cast<int>(phi) / 2) % n);
		d2 = static_cast<uint32_t>((dr2 + static_cast<int>(phi) / 2) % n);
		if (d1 > d2)
			std::swap(d1, d2);
	}
	// Histogram3D::getCoordsFromDetPair + getBinIdFromCoords (:366-417, :267-279).
	bool bin(uint32_t d1, uint32_t d2, uint64_t& out) const
	{
		if (d1 == 0 && d2 == 0)
			return false;
		if (d1 > d2)
			std::swap(d1, d2);
		uint32_t r1 = d1 % dpr, r2 = d2 % dpr;
		if (r1 > r2)
		{
			std::swap(d1, d2);
			std::swap(r1, r2);
		}
		const int64_t m = ringMap[static_cast<uint64_t>(r1) * dpr + r2];
		if (m < 0)
			return false;
		const uint64_t r_ring = m / dpr, phi = m % dpr;
		uint64_t doi1 = d1 / (rings * dpr), doi2 = d2 / (rings * dpr);
		if (r1 > r2)
			std::swap(doi1, doi2);
		const uint64_t r = r_ring * numDOIPoss + (doi1 + doi2 * ndoi);
		const int z1 = static_cast<int>((d1 / dpr) % rings);
		const int z2 = static_cast<int>((d2 / dpr) % rings);
		const uint64_t dz = static_cast<uint64_t>(std::abs(z2 - z1));
		if (dz > mrd)
			return false;
		const uint64_t removed = dz * (dz - 1) / 2;
		uint64_t zb = dz * rings + std::min(z1, z2) - removed;
		if (dz > 0 && z1 > z2)
			zb += numZBinDiff;
		out = zb * numPhi * numR + phi * numR + r;
		return true;
	}
	// Histogram3D::getDetPairFromCoords (:286-363).
	void pair(uint64_t binId, uint32_t& d1, uint32_t& d2) const
	{
		const uint64_t z_bin = binId / (numPhi * numR);
		const uint64_t phi = (binId % (numPhi * numR)) / numR;
		const uint64_t r = (binId % (numPhi * numR)) % numR;
		uint32_t a, b;
		pairInRing(r / numDOIPoss, phi, a, b);
		if (a == b)
		{
			d1 = d2 = 0;
			return;
		}
		const uint64_t doi_case = r % numDOIPoss;
		const uint64_t doi1 = doi_case % ndoi, doi2 = doi_case / ndoi;
		uint64_t z1, z2;
		if (z_bin < rings)
		{
			z1 = z2 = z_bin;
		}
		else
		{
			int cur = (static_cast<int>(z_bin) - static_cast<int>(rings)) % static_cast<int>(numZBinDiff) + static_cast<int>(rings);
			int planes = static_cast<int>(rings);
			uint64_t dz = 0;
			while (cur - planes >= 0)
			{
				cur -= planes;
				planes -= 1;
				dz++;
			}
			z1 = cur;
			z2 = z1 + dz;
			if (z_bin - rings >= numZBinDiff)
				std::swap(z1, z2);
		}
		d1 = static_cast<uint32_t>(a + z1 * dpr + doi1 * (dpr * rings));
		d2 = static_cast<uint32_t>(b + z2 * dpr + doi2 * (dpr * rings));
	}
};

int orc_histo3d_dims(const orc_scanner* s, uint64_t* dims)
{
	H3 h(s);
	dims[0] = h.numZBin;
	dims[1] = h.numPhi;
	dims[2] = h.numR;
	return 0;
}

int orc_histo3d_bins(const orc_scanner* s, uint64_t n, const uint32_t* d1,
                     const uint32_t* d2, uint64_t* bins)
{
	H3 h(s);
	for (uint64_t i = 0; i < n; i++)
		if (!h.bin(d1[i], d2[i], bins[i]))
			bins[i] = UINT64_MAX;
	return 0;
}

int orc_histo3d_detpairs(const orc_scanner* s, uint64_t n, const uint64_t* bins,
                         uint32_t* d1, uint32_t* d2)
{
	H3 h(s);
	for (uint64_t i = 0; i < n; i++)
		h.pair(bins[i], d1[i], d2[i]);
	return 0;
}

// convertToHistogram3D (ReconstructionUtils.cpp:659-720): values (nullable
// = 1) > 0 are added to their bin; d1 == d2 is skipped; pairs the reference
// would reject are counted in *n_invalid and skipped.
int orc_lm_to_histo3d(const orc_scanner* s, uint64_t n, const uint32_t* d1,
                      const uint32_t* d2, const float* values, float* histo,
                      uint64_t* n_invalid)
{
	H3 h(s);
	uint64_t bad = 0;
	for (uint64_t i = 0; i < n; i++)
	{
		const float v = values ? values[i] : 1.0f;
		if (!(v > 0))
			continue;
		if (d1[i] == d2[i])
			continue;
		uint64_t b;
		if (!h.bin(d1[i], d2[i], b))
		{
			bad++;
			continue;
		}
		histo[b] += v;
	}
	if (n_invalid)
		*n_invalid = bad;
	return 0;
}

int orc_tof_f32(float fwhm, int nstd, float lorNorm, float tof, float lo,
                float hi, float* out)
{
	Tof<float> t(fwhm, nstd);
	out[0] = t.weight(lorNorm, tof, lo, hi);
	t.alphaRange(out[1], out[2], lorNorm, tof);
	out[3] = t.sigma;
	out[4] = t.trunc;
	out[5] = t.norm;
	return 0;
}

}  // extern "C"

namespace orc
{
template <typename T>
struct ProjCtx
{
	Grid<T> g;
	std::unique_ptr<Tof<T>> tof;
	Psf psf;
	bool hasPsf = false;
	V3<T> off;
	const orc_proj* p;
	ProjCtx(const Image* im, const orc_proj* pp) : g(*im), p(pp)
	{
		off = {static_cast<T>(im->off_x), static_cast<T>(im->off_y), static_cast<T>(im->off_z)};
		if (pp->tof_fwhm_ps > 0)
			tof = std::make_unique<Tof<T>>(pp->tof_fwhm_ps, pp->tof_n_std);
		if (pp->psf_taps)
		{
			hasPsf = true;
			psf.num_s = pp->psf_num_s;
			psf.size = pp->psf_size;
			psf.sStep = pp->psf_s_step;
			psf.kSpacing = pp->psf_k_spacing;
			psf.taps = pp->psf_taps;
			psf.flipped.resize(psf.num_s * psf.size);
			for (int i = 0; i < psf.num_s; i++)
				for (int j = 0; j < psf.size; j++)
					psf.flipped[i * psf.size + psf.size - 1 - j] = psf.taps[i * psf.size + j];
		}
	}

	// Visits every (voxel, weight) of event i, ray by ray.  Returns the number
	// of rays (weights of multi-ray events still have to be divided by it).
	template <typename Visit, typename EndRay>
	void visitEvent(const float* lor, const float* orient, const float* tofv,
	                const float* rayOff, bool forward, Visit&& visit,
	                EndRay&& endRay) const
	{
		Ray<T> r{{T(lor[0]), T(lor[1]), T(lor[2])}, {T(lor[3]), T(lor[4]), T(lor[5])}};
		const float tv = tofv ? *tofv : 0.f;
		if (p->projector == 1)
		{
			const V3<T> o1{T(orient[0]), T(orient[1]), T(orient[2])};
			const V3<T> o2{T(orient[3]), T(orient[4]), T(orient[5])};
			dd<T>(g, sub(r.p1, off), sub(r.p2, off), o1, o2, p->crystal_trans,
			      p->crystal_z, tof.get(), tv, hasPsf ? &psf : nullptr, forward,
			      visit);
			endRay();
			return;
		}
		for (int k = 0; k < p->num_rays; k++)
		{
			Ray<T> rk = r;
			if (k > 0)
			{
				const V3<float> n1{orient[0], orient[1], orient[2]};
				const V3<float> n2{orient[3], orient[4], orient[5]};
				rk = offsetRay<T>(r, n1, n2, rayOff + (k - 1) * 4, p->crystal_z,
				                  p->crystal_trans);
			}
			const V3<T> a = sub(rk.p1, off), b = sub(rk.p2, off);
			if (tof)
			{
				if (p->incremental)
					siddon<T, true, true>(g, a, b, tof.get(), tv, visit);
				else
					siddon<T, false, true>(g, a, b, tof.get(), tv, visit);
			}
			else
			{
				if (p->incremental)
					siddon<T, true, false>(g, a, b, nullptr, tv, visit);
				else
					siddon<T, false, false>(g, a, b, nullptr, tv, visit);
			}
			endRay();
		}
	}
	template <typename Visit>
	void visitEvent(const float* lor, const float* orient, const float* tofv,
	                const float* rayOff, bool forward, Visit&& visit) const
	{
		visitEvent(lor, orient, tofv, rayOff, forward, visit, [] {});
	}
};

template <typename T>
int projectImpl(const Image* im, const orc_proj* p, uint64_t n, const float* lors,
                const float* orients, const float* tof, const int32_t* frames,
                const float* rayOffsets, const float* image_in, bool forward,
                T* values, T* image_out)
{
	ProjCtx<T> c(im, p);
	const int64_t V = im->nx * im->ny * im->nz;
	const int nr = (p->projector == 0) ? p->num_rays : 1;
	const int roStride = 4 * (nr - 1);
	if (forward)
	{
		parallelFor(n, p->threads, [&](size_t i, int)
		{
			const int fr = frames ? frames[i] : 0;
			if (fr < 0)
			{
				values[i] = 0;
				return;
			}
			const float* img = image_in + fr * V;
			// Per-ray partial sums added ray by ray, as
			// ProjectorSiddon::forwardProjection does (ProjectorSiddon.cpp:259-299).
			T acc = 0, ray = 0;
			c.visitEvent(lors + i * 6, orients ? orients + i * 6 : nullptr,
			             tof ? tof + i : nullptr,
			             rayOffsets ? rayOffsets + i * roStride : nullptr, true,
			             [&](int64_t o, T w) { ray += w * T(img[o]); },
			             [&] { acc += ray; ray = 0; });
			if (nr > 1)
				acc = acc / static_cast<T>(nr);
			values[i] = acc;
		});
		return 0;
	}
	// Back projection: per-thread accumulation images, summed at the end
	// (deterministic in double; order-free in float like the atomic path).
	const int threads = std::max(1, p->threads);
	const int64_t total = V * im->nt;
	std::vector<std::vector<T>> acc(threads, std::vector<T>(total, T(0)));
	parallelFor(n, threads, [&](size_t i, int t)
	{
		const int fr = frames ? frames[i] : 0;
		if (fr < 0)
			return;
		T* dst = acc[t].data() + fr * V;
		T v = values[i];
		if (nr > 1)
			v = v / static_cast<T>(nr);
		c.visitEvent(lors + i * 6, orients ? orients + i * 6 : nullptr,
		             tof ? tof + i : nullptr,
		             rayOffsets ? rayOffsets + i * roStride : nullptr, false,
		             [&](int64_t o, T w) { dst[o] += v * w; });
	});
	for (int t = 0; t < threads; t++)
		for (int64_t k = 0; k < total; k++)
			image_out[k] += acc[t][k];
	return 0;
}
}  // namespace orc

extern "C" {

// Forward (fwd=1) or back (fwd=0) projection of n LORs (6 floats each, scanner
// coordinates).  orients: 6 floats per event (needed by DD and multi-ray).
// ray_offsets: 4*(num_rays-1) uniforms in [-0.5,0.5] per event for rays >= 1.
// frames: per-event dynamic frame (nullable; < 0 skips the event).
int orc_project_f32(const Image* im, const orc_proj* p, uint64_t n,
                    const float* lors, const float* orients, const float* tof,
                    const int32_t* frames, const float* ray_offsets,
                    const float* image_in, int fwd, float* values,
                    float* image_out)
{
	return projectImpl<float>(im, p, n, lors, orients, tof, frames, ray_offsets,
	                          image_in, fwd != 0, values, image_out);
}

int orc_project_f64(const Image* im, const orc_proj* p, uint64_t n,
                    const float* lors, const float* orients, const float* tof,
                    const int32_t* frames, const float* ray_offsets,
                    const float* image_in, int fwd, double* values,
                    double* image_out)
{
	return projectImpl<double>(im, p, n, lors, orients, tof, frames,
	                           ray_offsets, image_in, fwd != 0, values,
	                           image_out);
}

// Voxel index sequence and weights of one single-ray Siddon LOR (float
// mirror).  Returns the number of crossings written (at most cap).
int64_t orc_siddon_trace_f32(const Image* im, const orc_proj* p,
                             const float* lor, float tof, int64_t* idx,
                             float* w, int64_t cap)
{
	ProjCtx<float> c(im, p);
	int64_t k = 0;
	c.visitEvent(lor, nullptr, p->tof_fwhm_ps > 0 ? &tof : nullptr, nullptr,
	             true,
	             [&](int64_t o, float ww)
	             {
		             if (k < cap)
		             {
			             idx[k] = o;
			             w[k] = ww;
		             }
		             k++;
	             });
	return k;
}

int64_t orc_siddon_trace_f64(const Image* im, const orc_proj* p,
                             const float* lor, float tof, int64_t* idx,
                             double* w, int64_t cap)
{
	ProjCtx<double> c(im, p);
	int64_t k = 0;
	c.visitEvent(lor, nullptr, p->tof_fwhm_ps > 0 ? &tof : nullptr, nullptr,
	             true,
	             [&](int64_t o, double ww)
	             {
		             if (k < cap)
		             {
			             idx[k] = o;
			             w[k] = ww;
		             }
		             k++;
	             });
	return k;
}

// One EM subset pass in the order of OSEM_CPU::computeEMUpdateImage
// (OSEM_CPU.cpp:329-374), per event: u = A x; u *= sens; u *= att;
// u *= global; u += additive; if |u| > thr: u = m/u * sens * att * global and
// accumulate A^T u into em_out (nt frames).  Optional arrays are nullable.
int orc_em_step_f64(const Image* im, const orc_proj* p, uint64_t n,
                    const float* lors, const float* orients, const float* tof,
                    const int32_t* frames, const float* ray_offsets,
                    const float* measurement, const float* sens,
                    const float* att, const float* additive, float global,
                    float denom_thr, const float* image_in, double* em_out)
{
	ProjCtx<double> c(im, p);
	const int64_t V = im->nx * im->ny * im->nz;
	const int nr = (p->projector == 0) ? p->num_rays : 1;
	const int roStride = 4 * (nr - 1);
	const int threads = std::max(1, p->threads);
	const int64_t total = V * im->nt;
	std::vector<std::vector<double>> acc(threads, std::vector<double>(total, 0.0));
	parallelFor(n, threads, [&](size_t i, int t)
	{
		const int fr = frames ? frames[i] : 0;
		if (fr < 0)
			return;
		const float* img = image_in + fr * V;
		const float* lor = lors + i * 6;
		const float* ori = orients ? orients + i * 6 : nullptr;
		const float* tv = tof ? tof + i : nullptr;
		const float* ro = ray_offsets ? ray_offsets + i * roStride : nullptr;
		double u = 0, ray = 0;
		c.visitEvent(lor, ori, tv, ro, true, [&](int64_t o, double w) { ray += w * img[o]; },
		             [&] { u += ray; ray = 0; });
		if (nr > 1)
			u /= nr;
		const double s = sens ? sens[i] : 1.0, a = att ? att[i] : 1.0;
		u *= s;
		u *= a;
		u *= global;
		if (additive)
			u += additive[i];
		if (std::abs(u) > denom_thr)
		{
			const double m = measurement ? measurement[i] : 1.0;
			u = m / u * s * a * global;
			if (nr > 1)
				u /= nr;
			double* dst = acc[t].data() + fr * V;
			c.visitEvent(lor, ori, tv, ro, false, [&](int64_t o, double w) { dst[o] += u * w; });
		}
	});
	for (int t = 0; t < threads; t++)
		for (int64_t k = 0; k < total; k++)
			em_out[k] += acc[t][k];
	return 0;
}

}  // extern "C"

// Image-space PSF: separable convolution along x, then y, then z, with
// circular borders and sums in tap order, out[i] = sum_kk k[kk + c] *
// in[circ(i - kk)], kk = -c..c (OperatorPsf::convolve,
// src/operators/OperatorPsf.cpp:288-375; util::circular, src/utils/Tools.cpp:160-167).
// T = float mirrors the reference's FP32 sums; T = double is the FP64 oracle.
template <typename T>
static void psfConvolve(int64_t nx, int64_t ny, int64_t nz, int64_t nt,
                        const float* in, T* out, const float* kx, int nkx,
                        const float* ky, int nky, const float* kz, int nkz,
                        bool flip)
{
	auto tap = [&](const float* k, int n, int j) -> T
	{ return static_cast<T>(flip ? k[n - 1 - j] : k[j]); };
	auto circ = [](int64_t M, int64_t x) { return x < 0 ? x + M : (x >= M ? x - M : x); };
	const int64_t V = nx * ny * nz;
	std::vector<T> a(V), b(V);
	for (int64_t t = 0; t < nt; t++)
	{
		const float* src = in + t * V;
		T* dst = out + t * V;
		const int cx = nkx / 2, cy = nky / 2, cz = nkz / 2;
		for (int64_t z = 0; z < nz; z++)
			for (int64_t y = 0; y < ny; y++)
				for (int64_t x = 0; x < nx; x++)
				{
					T sum = 0;
					for (int kk = -cx; kk <= cx; kk++)
						sum += tap(kx, nkx, kk + cx) *
						       static_cast<T>(src[(z * ny + y) * nx + circ(nx, x - kk)]);
					a[(z * ny + y) * nx + x] = sum;
				}
		for (int64_t z = 0; z < nz; z++)
			for (int64_t x = 0; x < nx; x++)
				for (int64_t y = 0; y < ny; y++)
				{
					T sum = 0;
					for (int kk = -cy; kk <= cy; kk++)
						sum += tap(ky, nky, kk + cy) * a[(z * ny + circ(ny, y - kk)) * nx + x];
					b[(z * ny + y) * nx + x] = sum;
				}
		for (int64_t x = 0; x < nx; x++)
			for (int64_t y = 0; y < ny; y++)
				for (int64_t z = 0; z < nz; z++)
				{
					T sum = 0;
					for (int kk = -cz; kk <= cz; kk++)
						sum += tap(kz, nkz, kk + cz) * b[(circ(nz, z - kk) * ny + y) * nx + x];
					dst[(z * ny + y) * nx + x] = sum;
				}
	}
}

extern "C" {

int orc_psf_convolve_f32(int64_t nx, int64_t ny, int64_t nz, int64_t nt,
                         const float* in, float* out, const float* kx, int nkx,
                         const float* ky, int nky, const float* kz, int nkz,
                         int adjoint)
{
	psfConvolve<float>(nx, ny, nz, nt, in, out, kx, nkx, ky, nky, kz, nkz, adjoint != 0);
	return 0;
}

int orc_psf_convolve_f64(int64_t nx, int64_t ny, int64_t nz, int64_t nt,
                         const float* in, double* out, const float* kx, int nkx,
                         const float* ky, int nky, const float* kz, int nkz,
                         int adjoint)
{
	psfConvolve<double>(nx, ny, nz, nt, in, out, kx, nkx, ky, nky, kz, nkz, adjoint != 0);
	return 0;
}

}  // extern "C"
