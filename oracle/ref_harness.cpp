// Test infrastructure, not product code.
//
// C-ABI harness over the YRT-PET 2.0.7 reference library compiled from its own
// sources.  Every entry point drives the reference's public C++ API on plain
// arrays so that tests and the CPU-baseline leg of bench.py can run the
// reference itself on the same inputs as the CUDA path.  Nothing here is
// linked into or called by the product library.
//
// The file is built twice:
//   oracle/ref.mk       -> oracle/_ref/libyrtref_harness.so, against the CPU
//                          library (OSEM entry points create OSEM_CPU, the
//                          list-mode projection runs OperatorProjector);
//   oracle/ref_cuda.mk  -> oracle/_ref_cuda/libyrtref_gpu_harness.so, with
//                          REF_HARNESS_GPU defined, against the library built
//                          with BUILD_CUDA: the same OSEM and list-mode
//                          projection entry points run the reference's GPU
//                          path (OSEM_GPU, OperatorProjectorDevice and its
//                          CUDA kernels);
//   oracle/ref_cuda.mk  -> oracle/_ref_cuda/libyrtref_b200_harness.so, with
//                          REF_HARNESS_B200 defined as well: the reference's
//                          drivers run on the product's binding classes
//                          (yrt-pet_b200/binding: OSEM_GPU_B200 and
//                          OperatorProjectorB200 over libyrtb), which is how
//                          the tests check that binding end to end.
//
// Reference interfaces exercised (paths inside the yrt-pet project):
//   Scanner ctor + DetRegular LUT   src/datastruct/scanner/Scanner.cpp:102-127,
//                                   src/datastruct/scanner/DetRegular.cpp:113-183
//   Histogram3D maps                src/datastruct/projection/Histogram3D.cpp:165-450
//   ProjectorSiddon                 src/operators/ProjectorSiddon.cpp:239-767
//   ProjectorDD                     src/operators/ProjectorDD.cpp:185-578
//   TimeOfFlightHelper              include/yrt-pet/operators/TimeOfFlight.hpp:19-85
//   convertToHistogram3D            src/utils/ReconstructionUtils.cpp:659-800
//   OSEM (CPU)                      src/recon/OSEM.cpp:315-365, OSEM_CPU.cpp:127-403
//   LR updater, LREM (CPU)          src/operators/ProjectorUpdater.cpp:228-280,
//                                   src/recon/LREM.cpp, LREM_CPU.cpp

#include "yrt-pet/datastruct/image/Image.hpp"
#include "yrt-pet/datastruct/projection/DynamicFraming.hpp"
#include "yrt-pet/datastruct/projection/LORMotion.hpp"
#include "yrt-pet/datastruct/projection/Histogram3D.hpp"
#include "yrt-pet/datastruct/projection/ListModeLUT.hpp"
#include "yrt-pet/datastruct/projection/ProjectionList.hpp"
#include "yrt-pet/datastruct/projection/UniformHistogram.hpp"
#include "yrt-pet/datastruct/scanner/Scanner.hpp"
#include "yrt-pet/operators/OperatorPsf.hpp"
#include "yrt-pet/operators/OperatorVarPsf.hpp"
#include "yrt-pet/operators/ProjectionPsfManager.hpp"
#include "yrt-pet/operators/ProjectorDD.hpp"
#include "yrt-pet/operators/ProjectorParams.hpp"
#include "yrt-pet/operators/ProjectorSiddon.hpp"
#include "yrt-pet/operators/TimeOfFlight.hpp"
#include "yrt-pet/recon/LREM.hpp"
#include "yrt-pet/recon/OSEM.hpp"
#include "yrt-pet/utils/Globals.hpp"
#include "yrt-pet/utils/ReconstructionUtils.hpp"

#include <chrono>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

using namespace yrt;

#ifdef REF_HARNESS_GPU
constexpr bool kUseGPU = true;
#else
constexpr bool kUseGPU = false;
#endif

#ifdef REF_HARNESS_B200
#include "yrtb_yrtpet.cuh"
static int g_b200_precision = YRTB_MIRROR;
#endif

namespace
{
// The OSEM driver of this build: OSEM_CPU, OSEM_GPU, or OSEM_GPU_B200.
std::unique_ptr<OSEM> createDriver(const Scanner& sc)
{
#ifdef REF_HARNESS_B200
	return b200::createOSEM(sc, g_b200_precision);
#else
	return util::createOSEM(sc, kUseGPU);
#endif
}
}  // namespace

extern "C" {

struct ref_scanner_desc
{
	float axialFOV, crystalSize_z, crystalSize_trans, crystalDepth,
	    scannerRadius;
	uint64_t detsPerRing, numRings, numDOI, maxRingDiff, minAngDiff,
	    detsPerBlock;
};

struct ref_image_desc
{
	int64_t nx, ny, nz, nt;
	float length_x, length_y, length_z, off_x, off_y, off_z;
};

static char g_err[512];
const char* ref_last_error() { return g_err; }
}

namespace
{
std::unique_ptr<Scanner> makeScanner(const ref_scanner_desc* s)
{
	return std::make_unique<Scanner>(
	    "ref", s->axialFOV, s->crystalSize_z, s->crystalSize_trans,
	    s->crystalDepth, s->scannerRadius, s->detsPerRing, s->numRings,
	    s->numDOI, s->maxRingDiff, s->minAngDiff, s->detsPerBlock);
}

ImageParams makeParams(const ref_image_desc* d)
{
	return ImageParams(d->nx, d->ny, d->nz, d->length_x, d->length_y,
	                   d->length_z, d->off_x, d->off_y, d->off_z, d->nt);
}

std::unique_ptr<ImageOwned> makeImage(const ref_image_desc* d,
                                      const float* data)
{
	auto img = std::make_unique<ImageOwned>(makeParams(d));
	img->allocate();
	const size_t n = d->nx * d->ny * d->nz * d->nt;
	if (data)
		std::memcpy(img->getRawPointer(), data, n * sizeof(float));
	else
		img->fill(0.0f);
	return img;
}

template <typename F>
int guarded(F&& f)
{
	try
	{
		f();
		return 0;
	}
	catch (const std::exception& e)
	{
		std::snprintf(g_err, sizeof(g_err), "%s", e.what());
		return 1;
	}
}

template <typename F>
void parallelFor(size_t n, int threads, F&& f)
{
	if (threads <= 1 || n < 1024)
	{
		for (size_t i = 0; i < n; i++)
			f(i, 0);
		return;
	}
	std::vector<std::thread> pool;
	const size_t chunk = (n + threads - 1) / threads;
	for (int t = 0; t < threads; t++)
	{
		pool.emplace_back(
		    [&, t]()
		    {
			    const size_t b = t * chunk, e = std::min(n, b + chunk);
			    for (size_t i = b; i < e; i++)
				    f(i, t);
		    });
	}
	for (auto& th : pool)
		th.join();
}
}  // namespace

extern "C" {

int ref_set_threads(int n)
{
	globals::setNumThreads(n);
	return 0;
}

// Crystal centres and orientations: out[d*6 + {0..5}] = x,y,z,nx,ny,nz.
int ref_scanner_lut(const ref_scanner_desc* s, float* out)
{
	return guarded(
	    [&]
	    {
		    auto sc = makeScanner(s);
		    for (size_t d = 0; d < sc->getNumDets(); d++)
		    {
			    const Vector3D p = sc->getDetectorPos(d);
			    const Vector3D n = sc->getDetectorOrient(d);
			    out[d * 6 + 0] = p.x;
			    out[d * 6 + 1] = p.y;
			    out[d * 6 + 2] = p.z;
			    out[d * 6 + 3] = n.x;
			    out[d * 6 + 4] = n.y;
			    out[d * 6 + 5] = n.z;
		    }
	    });
}

int ref_histo3d_dims(const ref_scanner_desc* s, uint64_t* dims)
{
	return guarded(
	    [&]
	    {
		    auto sc = makeScanner(s);
		    Histogram3DOwned h(*sc);
		    dims[0] = h.numZBin;
		    dims[1] = h.numPhi;
		    dims[2] = h.numR;
	    });
}

// bin id per detector pair; UINT64_MAX where the reference throws.
int ref_histo3d_bins(const ref_scanner_desc* s, uint64_t n, const uint32_t* d1,
                     const uint32_t* d2, uint64_t* bins)
{
	return guarded(
	    [&]
	    {
		    auto sc = makeScanner(s);
		    Histogram3DOwned h(*sc);
		    for (uint64_t i = 0; i < n; i++)
		    {
			    try
			    {
				    bins[i] = h.getBinIdFromDetPair(d1[i], d2[i]);
			    }
			    catch (const std::exception&)
			    {
				    bins[i] = UINT64_MAX;
			    }
		    }
	    });
}

int ref_histo3d_detpairs(const ref_scanner_desc* s, uint64_t n,
                         const uint64_t* bins, uint32_t* d1, uint32_t* d2)
{
	return guarded(
	    [&]
	    {
		    auto sc = makeScanner(s);
		    Histogram3DOwned h(*sc);
		    for (uint64_t i = 0; i < n; i++)
		    {
			    const det_pair_t p = h.getDetPairFromBinId(bins[i]);
			    d1[i] = p.d1;
			    d2[i] = p.d2;
		    }
	    });
}

// Sensitivity histogram of a normalisation made of crystal factors:
// out[bin] = eff[d1] * eff[d2] (FP32) for every bin of the scanner's
// Histogram3D, through the reference's own bin -> detector-pair map
// (Histogram3D::getDetPairFromBinId), on `threads` host threads.
int ref_histo3d_crystal_product(const ref_scanner_desc* s, const float* eff,
                                int threads, float* out)
{
	return guarded(
	    [&]
	    {
		    auto sc = makeScanner(s);
		    Histogram3DOwned h(*sc);
		    parallelFor(h.count(), threads,
		                [&](size_t b, int)
		                {
			                const det_pair_t p = h.getDetPairFromBinId(b);
			                out[b] = eff[p.d1] * eff[p.d2];
		                });
	    });
}

int ref_tof(float fwhm_ps, int n_std, float lorNorm, float tof_ps, float lo,
            float hi, float* out /* weight, amin, amax, sigma, trunc, norm */)
{
	TimeOfFlightHelper h(fwhm_ps, n_std);
	out[0] = h.getWeight(lorNorm, tof_ps, lo, hi);
	h.getAlphaRange(out[1], out[2], lorNorm, tof_ps);
	out[3] = h.getSigma();
	out[4] = h.getTruncWidth();
	out[5] = h.getNorm();
	return 0;
}

// Siddon forward (fwd=1: values[i] = A_i x) or back projection (fwd=0:
// image += A_i^T values[i]) of n arbitrary LORs (6 floats each).
// incr=1 uses the projector member path (offset subtracted, multi-ray
// capable); incr=0 uses the slow explicit instantiation on offset-subtracted
// LORs (single ray only).
int ref_siddon(const ref_scanner_desc* s, const ref_image_desc* d, float* image,
               uint64_t n, const float* lors, const float* orients,
               const float* tof, float tof_fwhm_ps, int tof_n_std,
               const int32_t* frames, int num_rays, int fwd, int incr,
               int threads, float* values)
{
	return guarded(
	    [&]
	    {
		    auto sc = makeScanner(s);
		    auto img = makeImage(d, image);
		    ProjectorParams pp(*sc);
		    pp.numRays = num_rays;
		    globals::setNumThreads(threads);
		    ProjectorSiddon proj(pp);
		    std::unique_ptr<TimeOfFlightHelper> tofh;
		    if (tof)
			    tofh = std::make_unique<TimeOfFlightHelper>(tof_fwhm_ps,
			                                                tof_n_std);
		    const Vector3D off{img->getParams().off_x, img->getParams().off_y,
		                       img->getParams().off_z};
		    parallelFor(
		        n, threads,
		        [&](size_t i, int tid)
		        {
			        Line3D lor{{lors[i * 6 + 0], lors[i * 6 + 1], lors[i * 6 + 2]},
			                   {lors[i * 6 + 3], lors[i * 6 + 4], lors[i * 6 + 5]}};
			        Vector3D n1{}, n2{};
			        if (orients)
			        {
				        n1 = {orients[i * 6 + 0], orients[i * 6 + 1],
				              orients[i * 6 + 2]};
				        n2 = {orients[i * 6 + 3], orients[i * 6 + 4],
				              orients[i * 6 + 5]};
			        }
			        const frame_t fr = frames ? frames[i] : 0;
			        const float tv = tof ? tof[i] : 0.f;
			        if (fr < 0)
			        {
				        if (fwd)
					        values[i] = 0.f;
				        return;
			        }
			        if (incr)
			        {
				        if (fwd)
					        values[i] = proj.forwardProjection(
					            img.get(), lor, n1, n2, tid, fr, tofh.get(), tv);
				        else
					        proj.backProjection(img.get(), lor, n1, n2, values[i],
					                            tid, fr, tofh.get(), tv);
			        }
			        else
			        {
				        lor.point1 = lor.point1 - off;
				        lor.point2 = lor.point2 - off;
				        float v = fwd ? 0.f : values[i];
				        if (tofh)
				        {
					        if (fwd)
						        ProjectorSiddon::project_helper<true, false, true,
						                                        false>(
						            img.get(), lor, v, nullptr, fr, tid,
						            tofh.get(), tv);
					        else
						        ProjectorSiddon::project_helper<false, false, true,
						                                        false>(
						            img.get(), lor, v, nullptr, fr, tid,
						            tofh.get(), tv);
				        }
				        else
				        {
					        if (fwd)
						        ProjectorSiddon::project_helper<true, false,
						                                        false, false>(
						            img.get(), lor, v, nullptr, fr, tid);
					        else
						        ProjectorSiddon::project_helper<false, false,
						                                        false, false>(
						            img.get(), lor, v, nullptr, fr, tid);
				        }
				        if (fwd)
					        values[i] = v;
			        }
		        });
		    if (!fwd)
		    {
			    const size_t nv = d->nx * d->ny * d->nz * d->nt;
			    std::memcpy(image, img->getRawPointer(), nv * sizeof(float));
		    }
	    });
}

// Distance-driven forward/back projection (optionally TOF and with a
// projection-space PSF read from a CSV file).
int ref_dd(const ref_scanner_desc* s, const ref_image_desc* d, float* image,
           uint64_t n, const float* lors, const float* orients, const float* tof,
           float tof_fwhm_ps, int tof_n_std, const char* psf_csv, int fwd,
           int threads, float* values)
{
	return guarded(
	    [&]
	    {
		    auto sc = makeScanner(s);
		    auto img = makeImage(d, image);
		    ProjectorParams pp(*sc);
		    globals::setNumThreads(threads);
		    ProjectorDD proj(pp);
		    std::unique_ptr<TimeOfFlightHelper> tofh;
		    if (tof)
			    tofh = std::make_unique<TimeOfFlightHelper>(tof_fwhm_ps,
			                                                tof_n_std);
		    std::unique_ptr<ProjectionPsfManager> psf;
		    if (psf_csv && psf_csv[0])
			    psf = std::make_unique<ProjectionPsfManager>(psf_csv);
		    parallelFor(
		        n, threads,
		        [&](size_t i, int tid)
		        {
			        Line3D lor{{lors[i * 6 + 0], lors[i * 6 + 1], lors[i * 6 + 2]},
			                   {lors[i * 6 + 3], lors[i * 6 + 4], lors[i * 6 + 5]}};
			        Vector3D n1{orients[i * 6 + 0], orients[i * 6 + 1],
			                    orients[i * 6 + 2]};
			        Vector3D n2{orients[i * 6 + 3], orients[i * 6 + 4],
			                    orients[i * 6 + 5]};
			        const float tv = tof ? tof[i] : 0.f;
			        if (fwd)
				        values[i] = proj.forwardProjection(img.get(), lor, n1, n2,
				                                           tid, 0, tofh.get(), tv,
				                                           psf.get());
			        else
				        proj.backProjection(img.get(), lor, n1, n2, values[i], tid,
				                            0, tofh.get(), tv, psf.get());
		        });
		    if (!fwd)
		    {
			    const size_t nv = d->nx * d->ny * d->nz * d->nt;
			    std::memcpy(image, img->getRawPointer(), nv * sizeof(float));
		    }
	    });
}

// Reads a ListModeLUT file with the reference reader; returns the number of
// events (or -1 on error) and fills the arrays when they are large enough.
int64_t ref_read_listmode(const ref_scanner_desc* s, const char* fname,
                          int tof, int randoms, uint64_t cap, uint32_t* ts,
                          uint32_t* d1, uint32_t* d2, float* tofv, float* rnd)
{
	int64_t n = -1;
	const int rc = guarded(
	    [&]
	    {
		    auto sc = makeScanner(s);
		    ListModeLUTOwned lm(*sc, fname, tof != 0, randoms != 0);
		    n = static_cast<int64_t>(lm.count());
		    for (uint64_t i = 0; i < std::min<uint64_t>(cap, lm.count()); i++)
		    {
			    ts[i] = lm.getTimestamp(i);
			    d1[i] = lm.getDetector1(i);
			    d2[i] = lm.getDetector2(i);
			    if (tof)
				    tofv[i] = lm.getTOFValue(i);
			    if (randoms)
				    rnd[i] = lm.getRandomsEstimate(i);
		    }
	    });
	return rc == 0 ? n : -1;
}

// Image-space PSF: OperatorPsf::applyA / applyAH (separable convolution with
// circular borders, src/operators/OperatorPsf.cpp:288-375).
int ref_psf_convolve(const ref_image_desc* d, const float* in, float* out,
                     const float* kx, int nkx, const float* ky, int nky,
                     const float* kz, int nkz, int adjoint)
{
	return guarded(
	    [&]
	    {
		    auto a = makeImage(d, in);
		    auto b = makeImage(d, nullptr);
		    OperatorPsf op(std::vector<float>(kx, kx + nkx),
		                   std::vector<float>(ky, ky + nky),
		                   std::vector<float>(kz, kz + nkz));
		    if (adjoint)
			    op.applyAH(a.get(), b.get());
		    else
			    op.applyA(a.get(), b.get());
		    const size_t n = d->nx * d->ny * d->nz * d->nt;
		    std::memcpy(out, b->getRawPointer(), n * sizeof(float));
	    });
}

// OperatorPsf::createGaussianKernel1D; size 0 = the reference's default.
int ref_psf_gaussian_kernel(float sigma, float vox, uint64_t size, float* out,
                            uint64_t cap, uint64_t* outSize)
{
	return guarded(
	    [&]
	    {
		    const size_t sz = size;
		    const auto k = OperatorPsf::createGaussianKernel1D(
		        sigma, vox, size ? &sz : nullptr);
		    *outSize = k.size();
		    for (size_t i = 0; i < k.size() && i < cap; i++)
			    out[i] = k[i];
	    });
}

float ref_dd_overlap(float p0, float p1, float d0, float d1)
{
	return ProjectorDD::getOverlap(p0, p1, d0, d1, nullptr, nullptr);
}

// List-mode -> Histogram3D binning (reference convertToHistogram3D with
// atomic accumulation).  histo must hold numZBin*numPhi*numR floats.
int ref_lm_to_histo3d(const ref_scanner_desc* s, uint64_t n, const uint32_t* d1,
                      const uint32_t* d2, int threads, float* histo,
                      double* seconds)
{
	return guarded(
	    [&]
	    {
		    auto sc = makeScanner(s);
		    globals::setNumThreads(threads);
		    ListModeLUTOwned lm(*sc);
		    lm.allocate(n);
		    for (uint64_t i = 0; i < n; i++)
			    lm.setDetectorIdsOfEvent(i, d1[i], d2[i]);
		    Histogram3DOwned h(*sc);
		    h.allocate();
		    h.clearProjections(0.0f);
		    const auto t0 = std::chrono::steady_clock::now();
		    util::convertToHistogram3D<true, false>(lm, h);
		    const auto t1 = std::chrono::steady_clock::now();
		    if (seconds)
			    *seconds = std::chrono::duration<double>(t1 - t0).count();
		    std::memcpy(histo, h.getData().getRawPointer(),
		                h.count() * sizeof(float));
	    });
}

struct ref_osem_desc
{
	int projector;  // 0 = Siddon, 1 = DD
	int num_rays;
	float tof_fwhm_ps;  // <= 0: no TOF
	int tof_n_std;
	int iterations;
	int subsets;
	int threads;
	float global_scale;
	float hard_threshold;
	int listmode;  // 1: list-mode events, 0: histogram input
	const char* image_psf_csv;  // image-space PSF (OSEM::addImagePSF), or NULL
	int image_psf_variant;      // 1: the CSV is a spatially variant PSF LUT
};

// Sensitivity image (reference OSEM::generateSensitivityImages).  sens_histo
// (nullable) is a Histogram3D of LOR sensitivities; att_image (nullable) is a
// hardware attenuation image on att_desc's grid.  Output: one image per subset
// (list-mode forces a single image), written back to back into out.
int ref_sensitivity(const ref_scanner_desc* s, const ref_image_desc* d,
                    const ref_osem_desc* o, const float* sens_histo,
                    const ref_image_desc* att_desc, const float* att_image,
                    const char* psf_csv, float* out, double* seconds)
{
	return guarded(
	    [&]
	    {
		    auto sc = makeScanner(s);
		    globals::setNumThreads(o->threads);
		    auto osem = createDriver(*sc);
		    osem->setImageParams(makeParams(d));
		    osem->num_OSEM_subsets = o->subsets;
		    osem->num_MLEM_iterations = o->iterations;
		    osem->hardThreshold = o->hard_threshold;
		    osem->setListModeEnabled(o->listmode != 0);
		    osem->setProjector(o->projector == 0 ? ProjectorType::SIDDON :
		                                           ProjectorType::DD);
		    osem->setNumRays(o->num_rays);
		    if (psf_csv && psf_csv[0])
			    osem->addProjPSF(psf_csv);
		    if (o->image_psf_csv && o->image_psf_csv[0])
			    osem->addImagePSF(o->image_psf_csv, o->image_psf_variant ?
			                                          ImagePSFMode::VARIANT :
			                                          ImagePSFMode::UNIFORM);
		    osem->setGlobalScalingFactor(o->global_scale);
		    std::unique_ptr<Histogram3DOwned> sh;
		    if (sens_histo)
		    {
			    sh = std::make_unique<Histogram3DOwned>(*sc);
			    sh->allocate();
			    std::memcpy(sh->getData().getRawPointer(), sens_histo,
			                sh->count() * sizeof(float));
			    osem->setSensitivityHistogram(sh.get());
		    }
		    std::unique_ptr<ImageOwned> att;
		    if (att_image)
		    {
			    att = makeImage(att_desc, att_image);
			    osem->setAttenuationImage(att.get());
		    }
		    std::vector<std::unique_ptr<Image>> sens;
		    const auto t0 = std::chrono::steady_clock::now();
		    osem->generateSensitivityImages(sens, "");
		    const auto t1 = std::chrono::steady_clock::now();
		    if (seconds)
			    *seconds = std::chrono::duration<double>(t1 - t0).count();
		    const size_t nv = d->nx * d->ny * d->nz;
		    for (size_t i = 0; i < sens.size(); i++)
			    std::memcpy(out + i * nv, sens[i]->getRawPointer(),
			                nv * sizeof(float));
	    });
}

// Optional list-mode extras: event timestamps, dynamic framing
// (numFrames+1 timestamps, DynamicFraming) and rigid LOR motion (LORMotion:
// starting timestamp + transform_t per motion frame).
struct ref_lm_extra
{
	const uint32_t* timestamps;
	uint64_t num_frame_ts;
	const uint32_t* frame_ts;
	uint64_t num_motion;
	const uint32_t* motion_starts;
	const float* motion;  // 12 floats per motion frame, transform_t order
};

// List-mode OSEM with the reference CPU path.  sens: one sensitivity image
// (list-mode).  Events: detector pairs, optional TOF (ps) and optional
// per-event additive (randoms) estimates.  Optional sensitivity histogram and
// attenuation image act as in the reference corrector.  out: nt images.
int ref_osem_listmode_ex(const ref_scanner_desc* s, const ref_image_desc* d,
                         const ref_osem_desc* o, const float* sens, uint64_t n,
                         const uint32_t* d1, const uint32_t* d2,
                         const float* tof, const float* randoms,
                         const float* sens_histo, const ref_image_desc* att_desc,
                         const float* att_image, const ref_lm_extra* ex,
                         float* out, double* seconds)
{
	return guarded(
	    [&]
	    {
		    auto sc = makeScanner(s);
		    globals::setNumThreads(o->threads);
		    ListModeLUTOwned lm(*sc, tof != nullptr, randoms != nullptr);
		    lm.allocate(n);
		    for (uint64_t i = 0; i < n; i++)
		    {
			    lm.setDetectorIdsOfEvent(i, d1[i], d2[i]);
			    if (tof)
				    lm.setTOFValueOfEvent(i, tof[i]);
			    if (randoms)
				    lm.setRandomsEstimateOfEvent(i, randoms[i]);
			    if (ex && ex->timestamps)
				    lm.setTimestampOfEvent(i, ex->timestamps[i]);
		    }
		    if (ex && ex->num_frame_ts > 1)
		    {
			    std::vector<timestamp_t> v(ex->frame_ts,
			                               ex->frame_ts + ex->num_frame_ts);
			    lm.addDynamicFraming(v);
		    }
		    if (ex && ex->num_motion > 0)
		    {
			    auto mot = std::make_shared<LORMotion>(ex->num_motion);
			    for (uint64_t f = 0; f < ex->num_motion; f++)
			    {
				    const float* m = ex->motion + f * 12;
				    transform_t t{m[0], m[1], m[2],  m[3],  m[4],  m[5],
				                  m[6], m[7], m[8], m[9], m[10], m[11]};
				    mot->setTransform(static_cast<frame_t>(f), t);
				    mot->setStartingTimestamp(static_cast<frame_t>(f),
				                              ex->motion_starts[f]);
			    }
			    lm.addLORMotion(mot);
		    }
		    auto osem = createDriver(*sc);
		    ImageParams ip = makeParams(d);
		    osem->setImageParams(ip);
		    osem->num_OSEM_subsets = o->subsets;
		    osem->num_MLEM_iterations = o->iterations;
		    osem->setListModeEnabled(true);
		    osem->setProjector(o->projector == 0 ? ProjectorType::SIDDON :
		                                           ProjectorType::DD);
		    osem->setNumRays(o->num_rays);
		    if (o->tof_fwhm_ps > 0)
			    osem->addTOF(o->tof_fwhm_ps, o->tof_n_std);
		    if (o->image_psf_csv && o->image_psf_csv[0])
			    osem->addImagePSF(o->image_psf_csv, o->image_psf_variant ?
			                                          ImagePSFMode::VARIANT :
			                                          ImagePSFMode::UNIFORM);
		    osem->setGlobalScalingFactor(o->global_scale);
		    std::unique_ptr<Histogram3DOwned> sh;
		    if (sens_histo)
		    {
			    sh = std::make_unique<Histogram3DOwned>(*sc);
			    sh->allocate();
			    std::memcpy(sh->getData().getRawPointer(), sens_histo,
			                sh->count() * sizeof(float));
			    osem->setSensitivityHistogram(sh.get());
		    }
		    std::unique_ptr<ImageOwned> att;
		    if (att_image)
		    {
			    att = makeImage(att_desc, att_image);
			    osem->setAttenuationImage(att.get());
		    }
		    ref_image_desc sd = *d;
		    sd.nt = 1;
		    auto sensImg = makeImage(&sd, sens);
		    osem->setSensitivityImage(sensImg.get(), 0);
		    osem->setDataInput(&lm);
		    const auto t0 = std::chrono::steady_clock::now();
		    auto res = osem->reconstruct("");
		    const auto t1 = std::chrono::steady_clock::now();
		    if (seconds)
			    *seconds = std::chrono::duration<double>(t1 - t0).count();
		    const ImageParams& rp = res->getParams();
		    const size_t nv = rp.nx * rp.ny * rp.nz * rp.nt;
		    std::memcpy(out, res->getRawPointer(), nv * sizeof(float));
	    });
}

int ref_osem_listmode(const ref_scanner_desc* s, const ref_image_desc* d,
                      const ref_osem_desc* o, const float* sens, uint64_t n,
                      const uint32_t* d1, const uint32_t* d2, const float* tof,
                      const float* randoms, const float* sens_histo,
                      const ref_image_desc* att_desc, const float* att_image,
                      float* out, double* seconds)
{
	return ref_osem_listmode_ex(s, d, o, sens, n, d1, d2, tof, randoms,
	                            sens_histo, att_desc, att_image, nullptr, out,
	                            seconds);
}

// Histogram-mode OSEM (measurements in a Histogram3D).
int ref_osem_histo3d(const ref_scanner_desc* s, const ref_image_desc* d,
                     const ref_osem_desc* o, const float* sens_images,
                     const float* histo, const char* psf_csv, float* out,
                     double* seconds)
{
	return guarded(
	    [&]
	    {
		    auto sc = makeScanner(s);
		    globals::setNumThreads(o->threads);
		    Histogram3DOwned h(*sc);
		    h.allocate();
		    std::memcpy(h.getData().getRawPointer(), histo,
		                h.count() * sizeof(float));
		    auto osem = createDriver(*sc);
		    osem->setImageParams(makeParams(d));
		    osem->num_OSEM_subsets = o->subsets;
		    osem->num_MLEM_iterations = o->iterations;
		    osem->setListModeEnabled(false);
		    osem->setProjector(o->projector == 0 ? ProjectorType::SIDDON :
		                                           ProjectorType::DD);
		    osem->setNumRays(o->num_rays);
		    if (psf_csv && psf_csv[0])
			    osem->addProjPSF(psf_csv);
		    if (o->image_psf_csv && o->image_psf_csv[0])
			    osem->addImagePSF(o->image_psf_csv, o->image_psf_variant ?
			                                          ImagePSFMode::VARIANT :
			                                          ImagePSFMode::UNIFORM);
		    if (o->tof_fwhm_ps > 0)
			    osem->addTOF(o->tof_fwhm_ps, o->tof_n_std);
		    const size_t nv = d->nx * d->ny * d->nz;
		    std::vector<std::unique_ptr<ImageOwned>> sensImgs;
		    for (int i = 0; i < o->subsets; i++)
		    {
			    sensImgs.push_back(makeImage(d, sens_images + i * nv));
			    osem->setSensitivityImage(sensImgs.back().get(), i);
		    }
		    osem->setDataInput(&h);
		    const auto t0 = std::chrono::steady_clock::now();
		    auto res = osem->reconstruct("");
		    const auto t1 = std::chrono::steady_clock::now();
		    if (seconds)
			    *seconds = std::chrono::duration<double>(t1 - t0).count();
		    std::memcpy(out, res->getRawPointer(), nv * sizeof(float));
	    });
}

// 1 when this build runs the reference's GPU path, 2 when it runs the
// reference's drivers on the libyrtb binding.
int ref_uses_gpu()
{
#ifdef REF_HARNESS_B200
	return 2;
#else
	return kUseGPU ? 1 : 0;
#endif
}

// Arithmetic of the libyrtb binding (YRTB_MIRROR or YRTB_COMPENSATED);
// other builds ignore it.
int ref_set_b200_precision(int precision)
{
#ifdef REF_HARNESS_B200
	g_b200_precision = precision;
#endif
	return 0;
}

// Forward (fwd=1: values[i] = A_i x) or back projection (fwd=0: image +=
// A^T values) of n list-mode events (detector pairs, optional TOF in ps)
// through util::forwProject / util::backProject
// (src/utils/ReconstructionUtils.cpp:948-1061) with one subset: the
// reference's OperatorProjector on the CPU build, OperatorProjectorDevice and
// its CUDA kernels (projectSiddon_kernel, projectDD_kernel) on the GPU build.
// o gives the projector (Siddon / DD), the number of rays, TOF and the host
// threads; psf_csv (nullable) a projection-space PSF.  On the GPU path the
// multi-ray offsets of event i are drawn with curand_init(13, i, 0)
// (include/yrt-pet/operators/SiddonKernels.cuh:27-84, 502-574) when all
// events fit one batch.
int ref_project_lm(const ref_scanner_desc* s, const ref_image_desc* d,
                   float* image, uint64_t n, const uint32_t* d1,
                   const uint32_t* d2, const float* tof, const ref_osem_desc* o,
                   const char* psf_csv, int fwd, float* values)
{
	return guarded(
	    [&]
	    {
		    auto sc = makeScanner(s);
		    globals::setNumThreads(o->threads);
		    ListModeLUTOwned lm(*sc, tof != nullptr, false);
		    lm.allocate(n);
		    for (uint64_t i = 0; i < n; i++)
		    {
			    lm.setDetectorIdsOfEvent(i, d1[i], d2[i]);
			    if (tof)
				    lm.setTOFValueOfEvent(i, tof[i]);
		    }
		    ProjectionListOwned pl(&lm);
		    pl.allocate();
		    if (fwd)
			    pl.clearProjections(0.0f);
		    else
			    std::memcpy(pl.getRawPointer(), values, n * sizeof(float));
		    ProjectorParams pp(*sc);
		    pp.projectorType =
		        o->projector == 0 ? ProjectorType::SIDDON : ProjectorType::DD;
		    pp.numRays = o->num_rays;
		    if (o->tof_fwhm_ps > 0)
			    pp.addTOF(o->tof_fwhm_ps, o->tof_n_std);
		    if (psf_csv && psf_csv[0])
			    pp.projPsf_fname = psf_csv;
		    auto img = makeImage(d, image);
		    const auto binIter = pl.getBinIter(1, 0);
#ifdef REF_HARNESS_B200
		    // The reference's operator contract on the binding's projector:
		    // OperatorProjectorDevice::applyA / applyAH stage the host data,
		    // batch it and call OperatorProjectorB200 per loaded batch.
		    std::vector<std::unique_ptr<Constraint>> cons;
		    sc->collectConstraints(cons);
		    std::vector<Constraint*> consPtr;
		    for (auto& c : cons)
			    consPtr.push_back(c.get());
		    auto op = b200::createOperatorProjectorDevice(
		        pp, binIter.get(), consPtr, nullptr, nullptr, g_b200_precision);
		    if (fwd)
			    op->applyA(img.get(), &pl);
		    else
			    op->applyAH(&pl, img.get());
#else
		    if (fwd)
			    util::forwProject(*img, pl, pp, *binIter, kUseGPU);
		    else
			    util::backProject(*img, pl, pp, *binIter, kUseGPU);
#endif
		    if (fwd)
		    {
			    std::memcpy(values, pl.getRawPointer(), n * sizeof(float));
		    }
		    else
		    {
			    const size_t nv = d->nx * d->ny * d->nz * d->nt;
			    std::memcpy(image, img->getRawPointer(), nv * sizeof(float));
		    }
	    });
}

// Incremental Siddon forward (fwd=1: values[i] = A x) or back projection
// (fwd=0: W += A^T values) of a low-rank image through the reference's
// ProjectorUpdaterLR: image holds rank frames W (d->nt = rank), H is
// rank x frames (row-major), frames[i] is each LOR's dynamic frame.
int ref_siddon_lr(const ref_scanner_desc* s, const ref_image_desc* d, float* image,
                  uint64_t n, const float* lors, const float* tof, float tof_fwhm_ps,
                  int tof_n_std, const int32_t* frames, float* H, int rank,
                  int num_frames, int fwd, int threads, float* values)
{
	return guarded(
	    [&]
	    {
		    auto sc = makeScanner(s);
		    auto img = makeImage(d, image);
		    ProjectorParams pp(*sc);
		    pp.updaterType = UpdaterType::LR;
		    pp.bindHBasis(H, rank, num_frames);
		    globals::setNumThreads(threads);
		    ProjectorSiddon proj(pp);
		    std::unique_ptr<TimeOfFlightHelper> tofh;
		    if (tof)
			    tofh = std::make_unique<TimeOfFlightHelper>(tof_fwhm_ps, tof_n_std);
		    const Vector3D zero{};
		    parallelFor(
		        n, threads,
		        [&](size_t i, int tid)
		        {
			        Line3D lor{{lors[i * 6 + 0], lors[i * 6 + 1], lors[i * 6 + 2]},
			                   {lors[i * 6 + 3], lors[i * 6 + 4], lors[i * 6 + 5]}};
			        const frame_t fr = frames[i];
			        const float tv = tof ? tof[i] : 0.f;
			        if (fwd)
				        values[i] = proj.forwardProjection(img.get(), lor, zero, zero,
				                                           tid, fr, tofh.get(), tv);
			        else
				        proj.backProjection(img.get(), lor, zero, zero, values[i], tid,
				                            fr, tofh.get(), tv);
		        });
		    if (!fwd)
		    {
			    const size_t nv = d->nx * d->ny * d->nz * d->nt;
			    std::memcpy(image, img->getRawPointer(), nv * sizeof(float));
		    }
	    });
}

// List-mode low-rank EM with the reference CPU path (LREM_CPU through
// util::createOSEM(scanner, false, true)): d->nt = rank; H (rank x frames,
// row-major) is bound as the HBasis and, with update_h, updated in place.
// timestamps / frame_ts give the events' dynamic frames (DynamicFraming with
// frames+1 boundaries).  init (nullable): initial W.  out: W (rank images).
int ref_lrem_listmode(const ref_scanner_desc* s, const ref_image_desc* d,
                      const ref_osem_desc* o, const float* sens, uint64_t n,
                      const uint32_t* d1, const uint32_t* d2, const float* tof,
                      const uint32_t* timestamps, const uint32_t* frame_ts,
                      float* H, int rank, int num_frames, int update_h,
                      const float* init, float* out, double* seconds)
{
	return guarded(
	    [&]
	    {
		    auto sc = makeScanner(s);
		    globals::setNumThreads(o->threads);
		    ListModeLUTOwned lm(*sc, tof != nullptr, false);
		    lm.allocate(n);
		    for (uint64_t i = 0; i < n; i++)
		    {
			    lm.setDetectorIdsOfEvent(i, d1[i], d2[i]);
			    if (tof)
				    lm.setTOFValueOfEvent(i, tof[i]);
			    lm.setTimestampOfEvent(i, timestamps[i]);
		    }
		    std::vector<timestamp_t> v(frame_ts, frame_ts + num_frames + 1);
		    lm.addDynamicFraming(v);
		    auto osem = util::createOSEM(*sc, false, true);
		    auto* lr = dynamic_cast<LREM*>(osem.get());
		    if (!lr)
			    throw std::runtime_error("createOSEM did not return an LREM");
		    ImageParams ip = makeParams(d);
		    osem->setImageParams(ip);
		    osem->num_OSEM_subsets = o->subsets;
		    osem->num_MLEM_iterations = o->iterations;
		    osem->setListModeEnabled(true);
		    osem->setProjector(o->projector == 0 ? ProjectorType::SIDDON :
		                                           ProjectorType::DD);
		    osem->setNumRays(o->num_rays);
		    if (o->tof_fwhm_ps > 0)
			    osem->addTOF(o->tof_fwhm_ps, o->tof_n_std);
		    osem->setGlobalScalingFactor(o->global_scale);
		    osem->setProjectorUpdaterType(UpdaterType::LR);
		    Array2DAlias<float> hb;
		    hb.bind(H, rank, num_frames);
		    lr->setHBasis(hb);
		    lr->setUpdateH(update_h != 0);
		    std::unique_ptr<ImageOwned> initImg;
		    if (init)
		    {
			    initImg = makeImage(d, init);
			    osem->setInitialEstimate(initImg.get());
		    }
		    ref_image_desc sd = *d;
		    sd.nt = 1;
		    auto sensImg = makeImage(&sd, sens);
		    osem->setSensitivityImage(sensImg.get(), 0);
		    osem->setDataInput(&lm);
		    const auto t0 = std::chrono::steady_clock::now();
		    auto res = osem->reconstruct("");
		    const auto t1 = std::chrono::steady_clock::now();
		    if (seconds)
			    *seconds = std::chrono::duration<double>(t1 - t0).count();
		    const ImageParams& rp = res->getParams();
		    const size_t nv = rp.nx * rp.ny * rp.nz * rp.nt;
		    std::memcpy(out, res->getRawPointer(), nv * sizeof(float));
	    });
}

// One kernel of the variant PSF LUT (ConvolutionKernelGaussian for
// columns = 3, ConvolutionKernelGaussianMixture for columns = 7).
int ref_varpsf_gaussian_kernel(const float* sig, int columns, const float* nstd,
                               const ref_image_desc* d, float* out, uint64_t cap,
                               int32_t* half_sizes, uint64_t* size)
{
	return guarded(
	    [&]
	    {
		    const ImageParams ip = makeParams(d);
		    std::unique_ptr<ConvolutionKernel> k;
		    if (columns == 7)
			    k = std::make_unique<ConvolutionKernelGaussianMixture>(
			        sig[0], sig[1], sig[2], sig[3], sig[4], sig[5], sig[6], nstd[0],
			        nstd[1], nstd[2], ip);
		    else
			    k = std::make_unique<ConvolutionKernelGaussian>(
			        sig[0], sig[1], sig[2], nstd[0], nstd[1], nstd[2], ip);
		    half_sizes[0] = static_cast<int32_t>(k->getHalfSizeX());
		    half_sizes[1] = static_cast<int32_t>(k->getHalfSizeY());
		    half_sizes[2] = static_cast<int32_t>(k->getHalfSizeZ());
		    const auto& a = k->getArray();
		    *size = a.getSizeTotal();
		    for (size_t i = 0; i < a.getSizeTotal() && i < cap; i++)
			    out[i] = a.getFlat(i);
	    });
}

// OperatorVarPsf(csv, params).applyA / applyAH into a zeroed output.
int ref_varpsf_apply(const ref_image_desc* d, const char* csv, const float* in, float* out,
                     int adjoint, int threads)
{
	return guarded(
	    [&]
	    {
		    globals::setNumThreads(threads);
		    auto src = makeImage(d, in);
		    auto dst = makeImage(d, nullptr);
		    OperatorVarPsf op(csv, makeParams(d));
		    if (adjoint)
			    op.applyAH(src.get(), dst.get());
		    else
			    op.applyA(src.get(), dst.get());
		    const size_t nv = d->nx * d->ny * d->nz * d->nt;
		    std::memcpy(out, dst->getRawPointer(), nv * sizeof(float));
	    });
}

}  // extern "C"
