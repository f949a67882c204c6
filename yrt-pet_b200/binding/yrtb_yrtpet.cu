/*
 * libyrtb inside YRT-PET's OperatorProjectorDevice and OSEM_GPU (see
 * yrtb_yrtpet.cuh).  Compiled against a YRT-PET source tree by
 * yrt-pet_b200/binding/binding.mk.
 */
#include "yrtb_yrtpet.cuh"

#include "yrt-pet/datastruct/image/ImageDevice.cuh"
#include "yrt-pet/datastruct/projection/ProjectionData.hpp"
#include "yrt-pet/datastruct/projection/ProjectionListDevice.cuh"
#include "yrt-pet/datastruct/scanner/Scanner.hpp"
#include "yrt-pet/geometry/Constants.hpp"
#include "yrt-pet/recon/Corrector_GPU.cuh"

#include <cuda_runtime.h>

#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>

namespace yrt::b200
{
namespace
{
void check(yrtb_status s)
{
	if (s != YRTB_OK)
		throw std::runtime_error(std::string("libyrtb: ") + yrtb_last_error());
}

void checkCuda(cudaError_t e, const char* what)
{
	if (e != cudaSuccess)
		throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// Projection-space PSF table in ProjectionPsfManager's CSV format
// (src/operators/ProjectionPsfManager.cpp:27-50): sStep, kSpacing,
// kernelSize, then numS * kernelSize taps, comma- or line-separated.
void readPsfCsv(const std::string& fname, yrtb_projector_params& p,
                std::vector<float>& taps)
{
	std::ifstream f(fname);
	if (!f)
		throw std::runtime_error("cannot open the projection PSF file " + fname);
	std::stringstream all;
	all << f.rdbuf();
	std::string text = all.str();
	for (char& c : text)
		if (c == '\n' || c == '\r')
			c = ',';
	std::vector<double> v;
	std::stringstream ss(text);
	std::string tok;
	while (std::getline(ss, tok, ','))
		if (tok.find_first_not_of(" \t") != std::string::npos)
			v.push_back(std::stod(tok));
	if (v.size() < 4)
		throw std::runtime_error("projection PSF file " + fname + " is too short");
	const int size = static_cast<int>(v[2]);
	if (size <= 0 || size % 2 == 0)
		throw std::runtime_error("Kernels must be of odd length");
	const size_t numS = (v.size() - 3) / static_cast<size_t>(size);
	taps.assign(v.begin() + 3, v.begin() + 3 + numS * size);
	p.psf_num_s = static_cast<int>(numS);
	p.psf_size = size;
	p.psf_s_step = static_cast<float>(v[0]);
	p.psf_k_spacing = static_cast<float>(v[1]);
	p.psf_taps = taps.data();
}

yrtb_image_params gridOf(const ImageParams& ip)
{
	return yrtb_image_params{ip.nx,       ip.ny,       ip.nz,      ip.nt,
	                         ip.length_x, ip.length_y, ip.length_z, ip.off_x,
	                         ip.off_y,    ip.off_z};
}

bool sameGrid(const ImageParams& a, const ImageParams& b)
{
	return a.nx == b.nx && a.ny == b.ny && a.nz == b.nz && a.nt == b.nt &&
	       a.length_x == b.length_x && a.length_y == b.length_y &&
	       a.length_z == b.length_z && a.off_x == b.off_x &&
	       a.off_y == b.off_y && a.off_z == b.off_z;
}
}  // namespace

// ----------------------------------------------------------------- Engine --
Engine::Engine(const ProjectorParams& pp, int precision)
{
	const Scanner& s = pp.scanner;
	m_scanner = yrtb_scanner{s.axialFOV,    s.crystalSize_z, s.crystalSize_trans,
	                         s.crystalDepth, s.scannerRadius, s.detsPerRing,
	                         s.numRings,    s.numDOI,        s.maxRingDiff,
	                         s.minAngDiff,  s.detsPerBlock};
	if (pp.updaterType != UpdaterType::DEFAULT4D)
		throw std::runtime_error("libyrtb projects with the DEFAULT4D updater "
		                         "only (the LR model runs through yrtb_lr_*)");
	m_params.projector =
	    pp.projectorType == ProjectorType::DD ? YRTB_DD : YRTB_SIDDON;
	m_params.num_rays = pp.projectorType == ProjectorType::DD ? 1 : pp.numRays;
	if (pp.hasTOF())
	{
		m_params.tof_fwhm_ps = pp.getTOFWidth_ps();
		m_params.tof_n_std = pp.getTOFNumStd();
	}
	if (!pp.projPsf_fname.empty())
		readPsfCsv(pp.projPsf_fname, m_params, m_psfTaps);
	m_params.precision = precision;
	m_params.deterministic = 0;
	m_buffers.assign(8, nullptr);
	m_capacity.assign(8, 0);
}

Engine::~Engine()
{
	if (m_proj)
		yrtb_projector_destroy(m_proj);
	for (void* b : m_buffers)
		if (b)
			cudaFree(b);
}

yrtb_projector* Engine::projector(const ImageParams& ip)
{
	if (m_proj && sameGrid(ip, m_projGrid))
		return m_proj;
	if (m_proj)
	{
		yrtb_projector_destroy(m_proj);
		m_proj = nullptr;
	}
	const yrtb_image_params g = gridOf(ip);
	check(yrtb_projector_create(&m_scanner, nullptr, &g, &m_params, &m_proj));
	m_projGrid = ip;
	return m_proj;
}

float* Engine::buffer(int which, size_t floats)
{
	if (m_capacity[which] < floats)
	{
		if (m_buffers[which])
			checkCuda(cudaFree(m_buffers[which]), "cudaFree");
		m_buffers[which] = nullptr;
		m_capacity[which] = 0;
		checkCuda(cudaMalloc(&m_buffers[which], floats * sizeof(float)),
		          "cudaMalloc of a batch buffer");
		m_capacity[which] = floats;
	}
	return static_cast<float*>(m_buffers[which]);
}

const yrtb_events& Engine::unpack(const PropertyUnit* d_rows, size_t n,
                                  const ProjectionPropertyManager& mgr,
                                  bool withCorrections, cudaStream_t stream)
{
	using P = ProjectionPropertyType;
	if (mgr.has(P::ATTENUATION_PRECORRECTION))
		throw std::runtime_error("libyrtb has no attenuation pre-correction "
		                         "factor per event");
	yrtb_row_layout L{};
	L.row_bytes = mgr.getElementSize();
	L.lor = mgr.getOffset(P::LOR);
	L.det_orient = mgr.getOffset(P::DET_ORIENT);
	L.tof = mgr.getOffset(P::TOF);
	L.dynamic_frame = mgr.getOffset(P::DYNAMIC_FRAME);
	L.measurement = mgr.getOffset(P::MEASUREMENT);
	L.sensitivity = mgr.getOffset(P::SENSITIVITY);
	L.attenuation = mgr.getOffset(P::ATTENUATION);
	L.randoms = mgr.getOffset(P::RANDOMS_ESTIMATE);
	L.scatter = mgr.getOffset(P::SCATTER_ESTIMATE);
	m_events = yrtb_events{};
	m_events.count = n;
	m_events.lor = buffer(0, 6 * n);
	if (mgr.has(P::DET_ORIENT))
		m_events.orient = buffer(1, 6 * n);
	if (mgr.has(P::TOF) && m_params.tof_fwhm_ps > 0.f)
		m_events.tof_ps = buffer(2, n);
	if (mgr.has(P::DYNAMIC_FRAME))
		m_events.frame = reinterpret_cast<const int32_t*>(buffer(3, n));
	if (withCorrections)
	{
		if (mgr.has(P::MEASUREMENT))
			m_events.measurement = buffer(4, n);
		if (mgr.has(P::SENSITIVITY))
			m_events.sens = buffer(5, n);
		if (mgr.has(P::ATTENUATION))
			m_events.att = buffer(6, n);
		if (mgr.has(P::RANDOMS_ESTIMATE) || mgr.has(P::SCATTER_ESTIMATE))
			m_events.additive = buffer(7, n);
	}
	check(yrtb_events_from_rows(d_rows, n, &L, &m_events,
	                            reinterpret_cast<yrtb_stream>(stream)));
	return m_events;
}

// ---------------------------------------------------- OperatorProjectorB200 --
OperatorProjectorB200::OperatorProjectorB200(
    const ProjectorParams& projParams, const BinIterator* binIter,
    const std::vector<Constraint*>& constraints, const cudaStream_t* mainStream,
    const cudaStream_t* auxStream, size_t memAvailable_bytes, int precision)
    : OperatorProjectorDevice(projParams, binIter, constraints, mainStream,
                              auxStream, memAvailable_bytes),
      m_engine(projParams, precision)
{
}

cudaStream_t OperatorProjectorB200::stream() const
{
	const cudaStream_t* s = getMainStream();
	return s ? *s : nullptr;
}

const ProjectionPropertyManager&
    OperatorProjectorB200::hostManager(const ProjectionListDevice& dat)
{
	// The batch's property manager lives on the device; it is a plain
	// structure (flags, element size, offsets), copied back per batch.
	checkCuda(cudaMemcpy(&m_manager, dat.getProjectionPropertyManagerDevicePointer(),
	                     sizeof(m_manager), cudaMemcpyDeviceToHost),
	          "reading the batch's property layout");
	return m_manager;
}

void OperatorProjectorB200::applyAOnLoadedBatch(ImageDevice& img,
                                                ProjectionListDevice& dat,
                                                bool synchronize)
{
	const size_t n = dat.getLoadedBatchSize();
	if (n == 0)
		return;
	const cudaStream_t st = stream();
	const yrtb_events& ev = m_engine.unpack(dat.getProjectionPropertiesDevicePointer(),
	                                        n, hostManager(dat), false, st);
	check(yrtb_forward(m_engine.projector(img.getParams()), img.getDevicePointer(),
	                   &ev, yrtb_range{0, 1, n}, dat.getProjValuesDevicePointer(),
	                   reinterpret_cast<yrtb_stream>(st)));
	if (synchronize)
		checkCuda(cudaStreamSynchronize(st), "forward projection");
}

void OperatorProjectorB200::applyAHOnLoadedBatch(ProjectionListDevice& dat,
                                                 ImageDevice& img,
                                                 bool synchronize)
{
	const size_t n = dat.getLoadedBatchSize();
	if (n == 0)
		return;
	const cudaStream_t st = stream();
	const yrtb_events& ev = m_engine.unpack(dat.getProjectionPropertiesDevicePointer(),
	                                        n, hostManager(dat), false, st);
	check(yrtb_backward(m_engine.projector(img.getParams()),
	                    dat.getProjValuesDevicePointer(), &ev, yrtb_range{0, 1, n},
	                    img.getDevicePointer(), reinterpret_cast<yrtb_stream>(st)));
	if (synchronize)
		checkCuda(cudaStreamSynchronize(st), "back projection");
}

// ------------------------------------------------------------ OSEM_GPU_B200 --
OSEM_GPU_B200::OSEM_GPU_B200(const Scanner& scanner, int precision)
    : OSEM_GPU(scanner), m_precision(precision)
{
}

void OSEM_GPU_B200::setupProjectorForRecon()
{
	OSEM_GPU::setupProjectorForRecon();
	mp_engine = std::make_unique<Engine>(projectorParams, m_precision);
}

void OSEM_GPU_B200::computeEMUpdateImage()
{
	auto* mlem = dynamic_cast<ImageDevice*>(getMLEMImageBuffer());
	auto* em = dynamic_cast<ImageDevice*>(getEMUpdateImageBuffer());
	if (!mlem || !em)
		throw std::runtime_error("OSEM_GPU_B200: device image buffers missing");
	// The image the subset's events are projected from: the MLEM image, or
	// its image-space PSF (OSEM_GPU::computeEMUpdateImage's forward PSF).
	ImageDevice* fwd = mlem;
	if (flagImagePSF)
	{
		mpd_tmpImage2->fill(0.0);
		imagePsf->applyA(mlem, mpd_tmpImage2.get());
		fwd = mpd_tmpImage2.get();
	}
	const cudaStream_t st = *getMainStream();
	const yrtb_stream yst = reinterpret_cast<yrtb_stream>(st);
	yrtb_projector* h = mp_engine->projector(fwd->getParams());
	const ProjectionPropertyManager& mgr = *mpd_propStruct->getManager();
	const float globalScale = mp_corrector->getGlobalScalingFactor();
	// Data without per-event measurements are uniform; the reference reads
	// their value from the first bin (OSEM_GPU.cu:900).
	const float uniform = getDataInput()->getProjectionValue(0);
	const bool needUniform =
	    !mgr.has(ProjectionPropertyType::MEASUREMENT) && uniform != 1.0f;
	std::vector<float> uniformHost;
	float* d_uniform = nullptr;

	const int subset = getCurrentOSEMSubset();
	for (int batch = 0; batch < getNumBatchesInSubset(subset); batch++)
	{
		precomputeBatchPropsForRecon(subset, batch);
		loadPrecomputedBatchPropsToDevice(subset, batch, {getMainStream(), true});
		const size_t n = getBatchSize(subset, batch);
		if (n == 0)
			continue;
		yrtb_events ev = mp_engine->unpack(mpd_propStruct->getDevicePointer(), n,
		                                   mgr, true, st);
		if (needUniform)
		{
			if (!d_uniform)
				checkCuda(cudaMallocAsync(reinterpret_cast<void**>(&d_uniform),
				                          getMaxBatchSize() * sizeof(float), st),
				          "cudaMallocAsync of the uniform measurements");
			check(yrtb_fill(d_uniform, n, uniform, yst));
			ev.measurement = d_uniform;
		}
		check(yrtb_em_step(h, fwd->getDevicePointer(), em->getDevicePointer(), &ev,
		                   yrtb_range{0, 1, n}, globalScale, denomThreshold, yst));
	}
	if (d_uniform)
		cudaFreeAsync(d_uniform, st);
	checkCuda(cudaStreamSynchronize(st), "EM pass");

	if (flagImagePSF)
	{
		// Adjoint PSF of the EM image into the update buffer.
		mpd_tmpImage2->fill(0.0);
		imagePsf->applyAH(em, mpd_tmpImage2.get());
		mpd_tmpImage1.swap(mpd_tmpImage2);
	}
}

void OSEM_GPU_B200::applyImageUpdate()
{
	auto* mlem = dynamic_cast<ImageDevice*>(getMLEMImageBuffer());
	auto* em = dynamic_cast<ImageDevice*>(getEMUpdateImageBuffer());
	auto* sens = dynamic_cast<ImageDevice*>(getSensImageBuffer());
	const ImageParams& ip = mlem->getParams();
	const uint64_t J = static_cast<uint64_t>(ip.nx) * ip.ny * ip.nz;
	// ImageDevice::updateEMThresholdDynamicDevice: static update for one
	// frame, else every frame against the first sensitivity frame (or a 4D
	// sensitivity image), threshold EPS_FLT.
	check(yrtb_em_update(mlem->getDevicePointer(), em->getDevicePointer(),
	                     sens->getDevicePointer(), J, ip.nt,
	                     sens->getParams().nt, EPS_FLT, nullptr,
	                     reinterpret_cast<yrtb_stream>(*getMainStream())));
	checkCuda(cudaStreamSynchronize(*getMainStream()), "EM update");
}

// -------------------------------------------------------------- factories --
std::unique_ptr<OperatorProjectorDevice> createOperatorProjectorDevice(
    const ProjectorParams& projParams, const BinIterator* binIter,
    const std::vector<Constraint*>& constraints, const cudaStream_t* mainStream,
    const cudaStream_t* auxStream, int precision)
{
	return std::make_unique<OperatorProjectorB200>(
	    projParams, binIter, constraints, mainStream, auxStream, 0, precision);
}

std::unique_ptr<OSEM> createOSEM(const Scanner& scanner, int precision)
{
	return std::make_unique<OSEM_GPU_B200>(scanner, precision);
}

}  // namespace yrt::b200
