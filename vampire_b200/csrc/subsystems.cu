// Context life-cycle hooks shared by the subsystems, kernel accounting and
// per-launch CUDA-event timing.
#include <cuda_runtime.h>

#include "vgpu_ctx.cuh"

using namespace vgpu;

int dipole_after_step(vgpu_ctx* h);
int dipole_ready(vgpu_ctx* h);

int vgpu_ctx::after_step() { return dipole_after_step(this); }
int vgpu_ctx::fields_ready() { return dipole_ready(this); }

void vgpu_ctx::destroy_extras() {
   stats_destroy(this);
   mc_destroy(this);
   dipole_destroy(this);
   batch_destroy(this);
   torque_destroy(this);
   cmc_destroy(this);
}

cudaEvent_t vgpu_ctx::get_event() {
   if (!event_pool.empty()) {
      cudaEvent_t e = event_pool.back();
      event_pool.pop_back();
      return e;
   }
   cudaEvent_t e = nullptr;
   if (cudaEventCreate(&e) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
   }
   return e;
}

void vgpu_ctx::prof_begin(int kind) {
   (void)kind;
   // sampled timing: the events between launches cost the stream a few
   // microseconds each and stop a staged pass from being scheduled early
   if (!prof_on || step % (uint64_t)prof_every != 0) return;
   prof_open = get_event();
   if (prof_open) cudaEventRecord(prof_open, stream);
}

void vgpu_ctx::prof_end(int kind) {
   if (!prof_on || !prof_open) return;
   cudaEvent_t b = get_event();
   if (!b) return;
   cudaEventRecord(b, stream);
   prof_pending.push_back({kind, prof_open, b});
   prof_open = nullptr;
   // keep the number of outstanding events bounded
   if (prof_pending.size() >= 4096) prof_collect();
}

int vgpu_ctx::prof_collect() {
   if (prof_pending.empty()) return VGPU_OK;
   cudaError_t e = cudaEventSynchronize(prof_pending.back().b);
   if (e != cudaSuccess) return cuda_err(this, e, "profile event");
   for (ProfRec& r : prof_pending) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
         prof_ms[r.kind] += ms;
         prof_count[r.kind] += 1;
      }
      event_pool.push_back(r.a);
      event_pool.push_back(r.b);
   }
   prof_pending.clear();
   return VGPU_OK;
}

extern "C" int vgpu_get_stream(vgpu_handle h, void** stream) {
   if (!h || !stream) return set_err(h, VGPU_ERR_ARG, "null argument");
   *stream = (void*)h->stream;
   return VGPU_OK;
}

extern "C" int vgpu_synchronize(vgpu_handle h) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   cudaSetDevice(h->device);
   int rc = cuda_err(h, cudaStreamSynchronize(h->stream), "synchronize");
   if (rc) return rc;
   return h->check_status();
}

extern "C" int vgpu_profile(vgpu_handle h, int enable) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   cudaSetDevice(h->device);
   int rc = h->prof_collect();
   for (int k = 0; k < PROF_KINDS; ++k) { h->prof_ms[k] = 0.0; h->prof_count[k] = 0; }
   h->kernel_launches = 0;
   h->prof_on = enable != 0;
   return rc;
}

extern "C" int vgpu_profile_read(vgpu_handle h, double* ms, int64_t* count, int32_t n_kinds, int64_t* kernel_launches) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   cudaSetDevice(h->device);
   int rc = h->prof_collect();
   if (rc) return rc;
   for (int k = 0; k < n_kinds && k < PROF_KINDS; ++k) {
      if (ms) ms[k] = h->prof_ms[k];
      if (count) count[k] = h->prof_count[k];
   }
   if (kernel_launches) *kernel_launches = h->kernel_launches;
   return VGPU_OK;
}
