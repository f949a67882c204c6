/*
 * libyrtb inside YRT-PET's own C++ classes.
 *
 * A maintainer adds these two classes (and the two factories) to a YRT-PET
 * build to run its existing drivers on libyrtb's kernels:
 *
 *   OperatorProjectorB200  an OperatorProjectorDevice
 *                          (include/yrt-pet/operators/OperatorProjectorDevice.cuh:20-97)
 *                          whose loaded batches are projected by yrtb_forward /
 *                          yrtb_backward instead of projectSiddon_kernel /
 *                          projectDD_kernel.  The base class keeps its own
 *                          host staging and batching (OperatorProjectorDevice::
 *                          applyA / applyAH, src/operators/OperatorProjectorDevice.cu:442-706).
 *   OSEM_GPU_B200          an OSEM_GPU (include/yrt-pet/recon/OSEM_GPU.cuh)
 *                          whose EM pass per subset (computeEMUpdateImage,
 *                          src/recon/OSEM_GPU.cu:455-510) runs yrtb_em_step on
 *                          every loaded batch and whose image update
 *                          (applyImageUpdate, OSEM_GPU.cu:512-516) runs
 *                          yrtb_em_update.  OSEM::reconstruct, the subsets,
 *                          the corrector, the batch loading and the
 *                          sensitivity images stay the reference's.
 *
 * The batches reach libyrtb as the reference keeps them on the device: one
 * packed row of projection properties per event
 * (PropStructManager<ProjectionPropertyType>); yrtb_events_from_rows unpacks
 * them into the structure of arrays the kernels read.  Errors are thrown as
 * std::runtime_error with libyrtb's message, as the reference's ASSERT_MSG
 * does.  Supported: Siddon (single and multi-ray), distance-driven with or
 * without a projection-space PSF, TOF, dynamic frames (DEFAULT4D).  The LR
 * updater and attenuation pre-correction factors are rejected (libyrtb runs
 * the LR model through yrtb_lr_*).
 */
#pragma once

#include "yrt_b200.h"

#include "yrt-pet/operators/OperatorProjectorDevice.cuh"
#include "yrt-pet/recon/OSEM_GPU.cuh"

#include <memory>
#include <vector>

namespace yrt::b200
{

// One libyrtb projector per image grid for one set of ProjectorParams, and
// the device arrays of the events of one batch.
class Engine
{
public:
	Engine(const ProjectorParams& params, int precision);
	~Engine();
	Engine(const Engine&) = delete;
	Engine& operator=(const Engine&) = delete;

	// The projector for this image grid (created on first use).
	yrtb_projector* projector(const ImageParams& ip);
	// Unpacks the n rows of a loaded batch (layout of the host copy of its
	// property manager) into this engine's event arrays; returns them.
	const yrtb_events& unpack(const PropertyUnit* d_rows, size_t n,
	                          const ProjectionPropertyManager& mgr,
	                          bool withCorrections, cudaStream_t stream);

private:
	float* buffer(int which, size_t floats);

	yrtb_scanner m_scanner{};
	yrtb_projector_params m_params{};
	std::vector<float> m_psfTaps;
	yrtb_projector* m_proj = nullptr;
	ImageParams m_projGrid;
	std::vector<void*> m_buffers;
	std::vector<size_t> m_capacity;
	yrtb_events m_events{};
};

class OperatorProjectorB200 : public OperatorProjectorDevice
{
public:
	explicit OperatorProjectorB200(
	    const ProjectorParams& projParams, const BinIterator* binIter = nullptr,
	    const std::vector<Constraint*>& constraints = {},
	    const cudaStream_t* mainStream = nullptr,
	    const cudaStream_t* auxStream = nullptr, size_t memAvailable_bytes = 0,
	    int precision = YRTB_MIRROR);

protected:
	void applyAOnLoadedBatch(ImageDevice& img, ProjectionListDevice& dat,
	                         bool synchronize) override;
	void applyAHOnLoadedBatch(ProjectionListDevice& dat, ImageDevice& img,
	                          bool synchronize) override;

private:
	const ProjectionPropertyManager& hostManager(const ProjectionListDevice& dat);
	cudaStream_t stream() const;

	Engine m_engine;
	const void* m_managerSource = nullptr;
	ProjectionPropertyManager m_manager{std::set<ProjectionPropertyType>{}};
};

class OSEM_GPU_B200 : public OSEM_GPU
{
public:
	explicit OSEM_GPU_B200(const Scanner& scanner, int precision = YRTB_MIRROR);

protected:
	void setupProjectorForRecon() override;
	void computeEMUpdateImage() override;
	void applyImageUpdate() override;

private:
	int m_precision;
	std::unique_ptr<Engine> mp_engine;
};

// util::createOperatorProjectorDevice (src/utils/ReconstructionUtilsDevice.cu:313)
// and util::createOSEM(scanner, true) (src/utils/ReconstructionUtils.cpp:915-933)
// returning the libyrtb classes.
std::unique_ptr<OperatorProjectorDevice> createOperatorProjectorDevice(
    const ProjectorParams& projParams, const BinIterator* binIter,
    const std::vector<Constraint*>& constraints = {},
    const cudaStream_t* mainStream = nullptr,
    const cudaStream_t* auxStream = nullptr, int precision = YRTB_MIRROR);
std::unique_ptr<OSEM> createOSEM(const Scanner& scanner,
                                 int precision = YRTB_MIRROR);

}  // namespace yrt::b200
