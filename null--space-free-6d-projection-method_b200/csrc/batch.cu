// Batched solves of independent Bloch points of uneven size (the batched Bloch
// path; the reference solves them one after another,
// exp4/run_exp4_medium.m:37-109).  Each instance gets its own context,
// stream, mass, basis and K_r^{-1} handles and runs the restarted Lanczos in
// its own host thread, so the GPU interleaves the kernels of small and large
// instances; the per-iteration PCG bodies replay captured CUDA graphs, and each
// instance may carry its own K_r^{-1} options (the schedule and pass tile shape the
// autotuner picked for its N).  Device memory is allocated stream-ordered from the
// library's pool on each instance's stream and every handle is released only after
// all instances finished, so no instance's free synchronises the device under the
// others.
#include <algorithm>
#include <cstring>
#include <string>
#include <thread>
#include <vector>
#include "internal.cuh"

using namespace fame;

namespace {

struct BatchJob {
  int device = 0, N = 0;
  const double* E = nullptr;
  double q[3] = {0, 0, 0};
  const double* P = nullptr;
  fame_krinv_opts o{};
  int nev = 0, maxiter = 0, p = 0;
  double tol = 0;
  unsigned long long seed = 0;
  double* theta = nullptr;
  fame_lanczos_info* info = nullptr;
  int status = FAME_OK;
  std::string error;
  fame_ctx* ctx = nullptr;
  fame_mass* m = nullptr;
  fame_basis* b = nullptr;
  fame_krinv* k = nullptr;
  void* v0 = nullptr;
};

// Set up and solve one instance on its own stream; the handles stay alive until
// every instance has finished (release_job), so that no instance frees device
// memory while others run.
void run_job(BatchJob* j) {
  int s = cudaSetDevice(j->device) == cudaSuccess ? FAME_OK : fail(FAME_ERR_CUDA, "cudaSetDevice");
  if (s == FAME_OK) s = fame_ctx_create(j->device, &j->ctx);
  if (s == FAME_OK) {
    StreamOrderedAlloc ordered(j->ctx->own);
    s = fame_mass_create(j->ctx, j->N, j->E, &j->m);
    if (s == FAME_OK) s = fame_basis_create(j->ctx, j->N, j->P, j->q, &j->b);
    if (s == FAME_OK) s = fame_krinv_create(j->b, j->m, &j->o, &j->k);
    if (s == FAME_OK) s = dalloc(&j->v0, 2 * (size_t)j->b->NF * sizeof(double2));
    if (s == FAME_OK) s = fame_start_vector(j->ctx, j->seed, 2 * j->b->NF, j->v0);
    if (s == FAME_OK) s = fame_lanczos(j->k, j->nev, j->tol, j->maxiter, j->p, j->v0, j->theta, nullptr, j->info);
    cudaStreamSynchronize(j->ctx->stream);
  }
  if (s != FAME_OK) j->error = fame_last_error();
  j->status = s;
}

void release_job(BatchJob* j) {
  if (!j->ctx) return;
  cudaSetDevice(j->device);
  StreamOrderedAlloc ordered(j->ctx->own);  // the context's workspace came from the pool too
  dfree(j->v0);
  fame_krinv_destroy(j->k);
  fame_basis_destroy(j->b);
  fame_mass_destroy(j->m);
  fame_ctx_destroy(j->ctx);
  j->ctx = nullptr;
}

}  // namespace

static int solve_batch(int device, int count, const int* Ns, const double* const* E, const double* q,
                       const double* P, const fame_krinv_opts* o, int per_instance, int nev, double tol,
                       int maxiter, int p, unsigned long long seed, double* theta, fame_lanczos_info* info,
                       int* status) {
  if (count < 1 || !Ns || !E || !q || !P || !theta || nev < 1 || (per_instance && !o))
    return fail(FAME_ERR_INVALID, "fame_solve_batch arguments");
  std::vector<BatchJob> jobs(count);
  for (int i = 0; i < count; ++i) {
    BatchJob& j = jobs[i];
    j.device = device;
    j.N = Ns[i];
    j.E = E[i];
    std::memcpy(j.q, q + 3 * i, sizeof(j.q));
    j.P = P;
    fame_krinv_default_opts(&j.o);
    if (o) j.o = per_instance ? o[i] : *o;
    j.nev = nev;
    j.tol = tol;
    j.maxiter = maxiter;
    j.p = p;
    j.seed = seed;
    j.theta = theta + (size_t)nev * i;
    j.info = info ? info + i : nullptr;
  }
  // the instances allocate from the library's own pool of the device, which keeps freed
  // blocks cached between the instances and across calls (mapping gigabytes anew costs
  // more than the small solves themselves); fame_device_trim_memory releases it
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return fail(FAME_ERR_CUDA, "fame_solve_batch: cannot select the device");
  }
  // largest instances first: they start their long chains of launches earliest
  std::vector<int> order(count);
  for (int i = 0; i < count; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return Ns[a] > Ns[b]; });
  std::vector<std::thread> threads;
  threads.reserve(count);
  for (int i : order) threads.emplace_back(run_job, &jobs[i]);
  for (auto& t : threads) t.join();
  for (int i = 0; i < count; ++i) release_job(&jobs[i]);
  cudaGetLastError();
  int first = FAME_OK;
  std::string msg;
  for (int i = 0; i < count; ++i) {
    if (status) status[i] = jobs[i].status;
    if (jobs[i].status != FAME_OK && first == FAME_OK) {
      first = jobs[i].status;
      msg = "instance " + std::to_string(i) + ": " + jobs[i].error;
    }
  }
  if (first != FAME_OK) return fail(first, msg);
  return FAME_OK;
}

extern "C" int fame_solve_batch(int device, int count, const int* Ns, const double* const* E,
                                const double* q, const double* P, const fame_krinv_opts* o, int nev,
                                double tol, int maxiter, int p, unsigned long long seed, double* theta,
                                fame_lanczos_info* info, int* status) {
  return solve_batch(device, count, Ns, E, q, P, o, 0, nev, tol, maxiter, p, seed, theta, info, status);
}

extern "C" int fame_solve_batch_each(int device, int count, const int* Ns, const double* const* E,
                                     const double* q, const double* P, const fame_krinv_opts* opts, int nev,
                                     double tol, int maxiter, int p, unsigned long long seed, double* theta,
                                     fame_lanczos_info* info, int* status) {
  return solve_batch(device, count, Ns, E, q, P, opts, 1, nev, tol, maxiter, p, seed, theta, info, status);
}
