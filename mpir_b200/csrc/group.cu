// Factor groups: several value sets on one analysed pattern refactorized by
// one CUDA graph launch.
//
// The reference factors one matrix per QDLDL_factor call (qdldl.hpp:172-345)
// and one GmresLDLIR per Compute.  Same-pattern instances (interior-point
// iterations, parameter sweeps) are independent factorizations over the same
// elimination tree: each member of a group is a solver on the shared plan
// with its own factor storage; the group records every member's
// factorization once, joins the recordings as parallel branches of one
// graph, and replays that graph for every new set of values.  Inside the
// launch the members' levels run concurrently, which fills the GPU where one
// factorization alone leaves SMs idle (the small fronts at the bottom of the
// tree, the chains of diagonal blocks at the top).  Each member is then
// solved as any solver (single or lockstep batched GMRES-IR).
#include <memory>
#include <vector>

#include "group.hpp"

namespace mpir {

FactorGroup::FactorGroup(Solver &base, int k) : device_(base.device) {
  if (k < 1) throw std::invalid_argument("a group holds at least one factor");
  if (!base.analyzed()) throw std::logic_error("group of a solver without an analysed pattern");
  MPIR_CUDA(cudaSetDevice(device_));
  MPIR_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  MPIR_CUDA(cudaEventCreate(&ev0_));
  MPIR_CUDA(cudaEventCreate(&ev1_));
  for (int i = 0; i < k; i++) {
    auto s        = std::make_unique<Solver>(base.uf, base.uw, base.ur, base.device);
    s->ir_iter    = base.ir_iter;
    s->gmres_iter = base.gmres_iter;
    s->tol        = base.tol;
    s->update_engine = base.update_engine;
    s->adopt(base.shared_plan());
    members_.push_back(std::move(s));
  }
}

FactorGroup::~FactorGroup() {
  cudaSetDevice(device_);
  if (stream_) cudaStreamSynchronize(stream_);
  if (exec_) cudaGraphExecDestroy(exec_);
  if (ev0_) cudaEventDestroy(ev0_);
  if (ev1_) cudaEventDestroy(ev1_);
  members_.clear();
  if (stream_) cudaStreamDestroy(stream_);
}

void FactorGroup::record() {
  cudaGraph_t parent = nullptr;
  MPIR_CUDA(cudaGraphCreate(&parent, 0));
  launches_ = 0;
  try {
    for (auto &m : members_) {
      int64_t           n     = 0;
      cudaGraph_t       child = m->record_factor(&n);
      cudaGraphNode_t   node;
      const cudaError_t e = cudaGraphAddChildGraphNode(&node, parent, nullptr, 0, child);
      cudaGraphDestroy(child);
      MPIR_CUDA(e);
      launches_ += n;
    }
    MPIR_CUDA(cudaGraphInstantiate(&exec_, parent, 0));
  } catch (...) {
    cudaGraphDestroy(parent);
    throw;
  }
  cudaGraphDestroy(parent);
}

int FactorGroup::factor(const double *Ax_host, int64_t stride, int64_t *npos) {
  MPIR_CUDA(cudaSetDevice(device_));
  const int64_t nnz = members_.front()->plan().S.nnz;
  // The members' value buffers are what the recording reads.
  for (size_t i = 0; i < members_.size(); i++)
    MPIR_CUDA(cudaMemcpyAsync(members_[i]->values_device(), Ax_host + i * stride,
                              nnz * sizeof(double), cudaMemcpyHostToDevice, stream_));
  if (!exec_) record();
  MPIR_CUDA(cudaEventRecord(ev0_, stream_));
  MPIR_CUDA(cudaGraphLaunch(exec_, stream_));
  launch_add(launches_);
  MPIR_CUDA(cudaEventRecord(ev1_, stream_));
  MPIR_CUDA(cudaEventSynchronize(ev1_));
  float ms = 0;
  MPIR_CUDA(cudaEventElapsedTime(&ms, ev0_, ev1_));
  last_ms_ = ms;
  int rc = kOk;
  for (size_t i = 0; i < members_.size(); i++) {
    const int r = members_[i]->finish_recorded_factor(ms);
    if (npos) npos[i] = members_[i]->last_npos;
    if (r != kOk && rc == kOk) rc = r;
  }
  return rc;
}

}  // namespace mpir
