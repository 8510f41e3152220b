// C ABI of the FoF library (include/cmh_fof.h): plans, one-shot runs,
// catalogs, errors.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <tuple>
#include <vector>

#include "cmh_internal.cuh"
#include "plan.cuh"

namespace cmh {

thread_local long long g_launches = 0;

namespace {
thread_local std::string g_last_error;

struct CatalogStore {
  bool host_owned = false;
};
}  // namespace

void set_error(const std::string &msg) { g_last_error = msg; }

void cuda_check(cudaError_t e, const char *what, const char *file, int line) {
  if (e == cudaSuccess) return;
  char buf[512];
  snprintf(buf, sizeof buf, "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
  throw Error{e == cudaErrorMemoryAllocation ? CMH_ERR_OUT_OF_MEMORY : CMH_ERR_CUDA, buf};
}

void fail(cmh_status code, const std::string &msg) { throw Error{code, msg}; }

bool fault_active(const char *kind) {
  const char *v = getenv("CMH_FAULT");
  if (!v || !*v) return false;
  const size_t n = strlen(kind);
  for (const char *p = v; *p;) {
    const char *e = strchr(p, ',');
    const size_t len = e ? (size_t)(e - p) : strlen(p);
    if (len == n && strncmp(p, kind, n) == 0) return true;
    if (!e) break;
    p = e + 1;
  }
  return false;
}

int resident_ctas(const void *kernel, int threads, size_t smem) {
  static std::mutex mu;
  static std::map<std::tuple<const void *, int, size_t, int>, int> cache;
  int dev = 0, sms = kSMs;
  CMH_CUDA(cudaGetDevice(&dev));
  const auto key = std::make_tuple(kernel, threads, smem, dev);
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  int per_sm = 0;
  CMH_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem));
  CMH_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int n = std::max(1, per_sm) * std::max(1, sms);
  cache[key] = n;
  return n;
}

void DevBuf::ensure(size_t bytes) {
  if (bytes <= cap && p) return;
  if (fault_active("alloc"))
    fail(CMH_ERR_OUT_OF_MEMORY, "device allocation failed (injected: CMH_FAULT=alloc)");
  if (p) CMH_CUDA(cudaFree(p));
  p = nullptr;
  cap = 0;
  size_t want = bytes + bytes / 64 + 256;  // headroom against small regrowth
  const cudaError_t e = cudaMalloc(&p, want);
  if (e == cudaErrorMemoryAllocation) {
    (void)cudaGetLastError();
    p = nullptr;
    fail(CMH_ERR_OUT_OF_MEMORY, "device memory exhausted (" + std::to_string(want >> 20) +
                                    " MiB requested)");
  }
  CMH_CUDA(e);
  cap = want;
}

void DevBuf::release() {
  if (p) cudaFree(p);
  p = nullptr;
  cap = 0;
}

Plan::Plan(const cmh_fof_params &p, int pdt, int dev) : device(dev), pos_dtype(pdt) {
  CMH_CUDA(cudaSetDevice(device));
  int major = 0;
  CMH_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
  if (major < 10) fail(CMH_ERR_NO_DEVICE, "the FoF kernels are built for sm_100a (B200)");
  CMH_CUDA(cudaEventCreate(&ev0));
  CMH_CUDA(cudaEventCreate(&ev1));
  for (cudaEvent_t &e : stage_ev) CMH_CUDA(cudaEventCreate(&e));
  set_params(p);
}

Plan::~Plan() {
  cudaSetDevice(device);
  for (cudaGraphExec_t g : graph_exec)
    if (g) cudaGraphExecDestroy(g);
  if (side_stream) cudaStreamSynchronize(side_stream);
  if (cap_stream) cudaStreamDestroy(cap_stream);
  if (bf_stream) {
    cudaStreamSynchronize(bf_stream);
    cudaStreamDestroy(bf_stream);
  }
  if (ev_fork) cudaEventDestroy(ev_fork);
  if (ev_join) cudaEventDestroy(ev_join);
  for (cudaEvent_t e : {ev_cleared, ev_emitted, ev_cleared2})
    if (e) cudaEventDestroy(e);
  if (side_stream) cudaStreamDestroy(side_stream);
  if (ev_side_start) cudaEventDestroy(ev_side_start);
  if (ev_pos_free) cudaEventDestroy(ev_pos_free);
  if (ev_vel_free) cudaEventDestroy(ev_vel_free);
  for (int b = 0; b < 2; b++) {
    if (ev_pos[b]) cudaEventDestroy(ev_pos[b]);
    if (ev_vel[b]) cudaEventDestroy(ev_vel[b]);
  }
  each_buf([](DevBuf &b) { b.release(); });
  if (ev0) cudaEventDestroy(ev0);
  if (ev1) cudaEventDestroy(ev1);
  for (cudaEvent_t e : stage_ev)
    if (e) cudaEventDestroy(e);
}

void Plan::release_workspace() {
  cudaSetDevice(device);
  for (int q = 0; q < 2; q++) {
    if (graph_exec[q]) cudaGraphExecDestroy(graph_exec[q]);
    graph_exec[q] = nullptr;
    graph_sig[q].clear();
  }
  if (side_stream) cudaStreamSynchronize(side_stream);
  staged.clear();
  uploaded_sig.clear();
  each_buf([](DevBuf &b) { b.release(); });
  np_cap = nd_cap = nc_cap = 0;
}

void Plan::set_params(const cmh_fof_params &p) {
  if (!(p.linklength > 0) || !(p.boundary >= 0))
    fail(CMH_ERR_INVALID_ARGUMENT, "Linklength must be > 0 and Boundarysize >= 0");
  if (p.precision != CMH_PLAIN_FP64 && p.precision != CMH_FP32_RECHECK)
    fail(CMH_ERR_INVALID_ARGUMENT, "unknown precision mode");
  params = p;
  fp32 = p.precision == CMH_FP32_RECHECK;
  ltab_host.clear();
  if (p.varlink) {
    if (p.ltab_n < 2 || !p.ltab || !(p.ltab_rmax > 0))
      fail(CMH_ERR_INVALID_ARGUMENT, "variable linking length needs a table of >= 2 entries");
    ltab_host.assign(p.ltab, p.ltab + p.ltab_n);
  }
  params.ltab = nullptr;  // the plan keeps its own copy
}

}  // namespace cmh

using cmh::Error;
using cmh::Plan;

#define CMH_API_BEGIN try {
#define CMH_API_END                                 \
  return CMH_OK;                                    \
  }                                                 \
  catch (const Error &e) {                          \
    cmh::set_error(e.msg);                          \
    return e.code;                                  \
  }                                                 \
  catch (const std::bad_alloc &) {                  \
    cmh::set_error("host allocation failed");       \
    return CMH_ERR_OUT_OF_MEMORY;                   \
  }                                                 \
  catch (const std::exception &e) {                 \
    cmh::set_error(e.what());                       \
    return CMH_ERR_INVALID_ARGUMENT;                \
  }

namespace {
// The caller's current device; CMH_ERR_NO_DEVICE when there is none (or no
// usable driver), rather than the runtime's error text.
int current_device() {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    (void)cudaGetLastError();
    cmh::fail(CMH_ERR_NO_DEVICE, "no usable CUDA device");
  }
  int dev = 0;
  CMH_CUDA(cudaGetDevice(&dev));
  return dev;
}

void check_parts(const cmh_particles *parts) {
  if (!parts) cmh::fail(CMH_ERR_INVALID_ARGUMENT, "particles is NULL");
  if (parts->n < 0) cmh::fail(CMH_ERR_INVALID_ARGUMENT, "negative particle count");
  if (parts->n > 0 && (!parts->pos || !parts->vel))
    cmh::fail(CMH_ERR_INVALID_ARGUMENT, "pos and vel are required");
  if ((parts->pos_dtype != CMH_FLOAT32 && parts->pos_dtype != CMH_FLOAT64) ||
      (parts->vel_dtype != CMH_FLOAT32 && parts->vel_dtype != CMH_FLOAT64))
    cmh::fail(CMH_ERR_INVALID_ARGUMENT, "unknown dtype");
  if (parts->n >= (int64_t)0xfffffff0ll)
    cmh::fail(CMH_ERR_CAPACITY, "more than 2^32 particles in one domain");
}

// Copies box b's part of the plan's last catalog to host arrays owned by
// `cat` (a run's catalog lists the boxes one after another).
void catalog_to_host(Plan &pl, cmh_catalog *cat, bool want_member, int b, cudaStream_t s) {
  const int nbox = (int)pl.boxes_host.size();
  const int64_t nh = pl.boxd_host[5 * nbox + b];
  const int64_t h0 = pl.boxd_host[6 * nbox + b];
  const int64_t n_in = pl.boxes_host[b].n;
  const int64_t i0 = (int64_t)pl.boxes_host[b].in_base;
  const int hs = pl.hs;
  cat->nhalos = nh;
  cat->halosize = hs;
  cat->location = CMH_HOST;
  cat->props = (float *)malloc(sizeof(float) * (size_t)std::max<int64_t>(nh * hs, 1));
  cat->head = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)std::max<int64_t>(nh, 1));
  cat->member = nullptr;
  cat->member_proc = nullptr;
  cat->member_pos = nullptr;
  cat->impl = new cmh::CatalogStore{true};
  if (want_member) {
    const size_t nn = (size_t)std::max<int64_t>(n_in, 1);
    cat->member = (int64_t *)malloc(sizeof(int64_t) * nn);
    cat->member_proc = (uint32_t *)malloc(sizeof(uint32_t) * nn);
    cat->member_pos = (float *)malloc(sizeof(float) * 3 * nn);
  }
  if (!cat->props || !cat->head ||
      (want_member && (!cat->member || !cat->member_proc || !cat->member_pos)))
    cmh::fail(CMH_ERR_OUT_OF_MEMORY, "host catalog allocation failed");
  if (nh > 0) {
    CMH_CUDA(cudaMemcpyAsync(cat->props, pl.b_props.as<float>() + h0 * hs,
                             sizeof(float) * nh * hs, cudaMemcpyDeviceToHost, s));
    CMH_CUDA(cudaMemcpyAsync(cat->head, pl.b_head_out.as<uint32_t>() + h0,
                             sizeof(uint32_t) * nh, cudaMemcpyDeviceToHost, s));
  }
  if (want_member && n_in > 0) {
    CMH_CUDA(cudaMemcpyAsync(cat->member, pl.b_member.as<int64_t>() + i0,
                             sizeof(int64_t) * n_in, cudaMemcpyDeviceToHost, s));
    CMH_CUDA(cudaMemcpyAsync(cat->member_proc, pl.b_member_proc.as<uint32_t>() + i0,
                             sizeof(uint32_t) * n_in, cudaMemcpyDeviceToHost, s));
    CMH_CUDA(cudaMemcpyAsync(cat->member_pos, pl.b_member_pos.as<float>() + 3 * i0,
                             sizeof(float) * 3 * n_in, cudaMemcpyDeviceToHost, s));
  }
  CMH_CUDA(cudaStreamSynchronize(s));
  if (want_member && h0 > 0)
    for (int64_t i = 0; i < n_in; i++)
      if (cat->member[i] >= 0) cat->member[i] -= h0;
  cat->stats = pl.stats;
  if (nbox > 1) {
    cat->stats.n_in = n_in;
    cat->stats.nhalos = nh;
    cat->stats.n_images = pl.boxd_host[3 * nbox + b];
    cat->stats.n_proc = (int64_t)pl.boxd_host[2 * nbox + b] + pl.boxd_host[3 * nbox + b];
    cat->stats.n_out = n_in - pl.boxd_host[2 * nbox + b];
  }
}

void catalog_on_device(Plan &pl, cmh_catalog *cat, bool want_member) {
  cat->nhalos = pl.out_nhalos;
  cat->halosize = pl.hs;
  cat->location = CMH_DEVICE;
  cat->props = pl.b_props.as<float>();
  cat->head = pl.b_head_out.as<uint32_t>();
  cat->member = want_member ? pl.b_member.as<int64_t>() : nullptr;
  cat->member_proc = want_member ? pl.b_member_proc.as<uint32_t>() : nullptr;
  cat->member_pos = want_member ? pl.b_member_pos.as<float>() : nullptr;
  cat->impl = nullptr;
  cat->stats = pl.stats;
}

}  // namespace

extern "C" {

int cmh_abi_version(void) { return CMH_ABI_VERSION; }

size_t cmh_last_error(char *buf, size_t len) {
  const std::string &m = cmh::g_last_error;
  if (buf && len) {
    size_t k = m.size() < len - 1 ? m.size() : len - 1;
    memcpy(buf, m.data(), k);
    buf[k] = 0;
  }
  return m.size();
}

cmh_status cmh_plan_create(cmh_plan **plan, const cmh_fof_params *params,
                           int64_t max_particles, int32_t pos_dtype, int32_t device) {
  CMH_API_BEGIN
  if (!plan || !params) cmh::fail(CMH_ERR_INVALID_ARGUMENT, "plan and params are required");
  *plan = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    cmh::fail(CMH_ERR_NO_DEVICE, "no CUDA device");
  if (device < 0 || device >= ndev) cmh::fail(CMH_ERR_INVALID_ARGUMENT, "bad device index");
  (void)max_particles;
  *plan = new Plan(*params, pos_dtype, device);
  CMH_API_END
}

cmh_status cmh_plan_set_params(cmh_plan *plan, const cmh_fof_params *params) {
  CMH_API_BEGIN
  if (!plan || !params) cmh::fail(CMH_ERR_INVALID_ARGUMENT, "plan and params are required");
  static_cast<Plan *>(plan)->set_params(*params);
  CMH_API_END
}

cmh_status cmh_plan_run(cmh_plan *plan, const cmh_particles *parts, cmh_catalog *cat,
                        int32_t want_member, int32_t out_location, void *stream) {
  CMH_API_BEGIN
  if (!plan || !cat) cmh::fail(CMH_ERR_INVALID_ARGUMENT, "plan and catalog are required");
  check_parts(parts);
  Plan &pl = *static_cast<Plan *>(plan);
  if (parts->pos_dtype != pl.pos_dtype)
    cmh::fail(CMH_ERR_INVALID_ARGUMENT, "position dtype differs from the plan's");
  memset(cat, 0, sizeof *cat);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cmh_particles dp = *parts;
  // host particles: copied into plan-owned device buffers on the plan's side
  // stream (or already being copied, by cmh_plan_prefetch)
  if (parts->location == CMH_HOST && parts->n > 0) dp = pl.take_inputs(parts, 1, s)[0];
  struct Reset {
    Plan &p;
    ~Reset() { p.vel_wait = false; }
  } reset{pl};
  pl.run(dp, want_member != 0, s);
  if (out_location == CMH_DEVICE) catalog_on_device(pl, cat, want_member != 0);
  else catalog_to_host(pl, cat, want_member != 0, 0, s);
  CMH_API_END
}

namespace {
void prefetch_on(Plan &pl, const cmh_particles *parts, int32_t nbox, void *stream) {
  int64_t total = 0;
  for (int b = 0; b < nbox; b++) {
    check_parts(&parts[b]);
    if (parts[b].location != CMH_HOST)
      cmh::fail(CMH_ERR_INVALID_ARGUMENT, "only host-resident particles are copied ahead");
    if (parts[b].pos_dtype != pl.pos_dtype)
      cmh::fail(CMH_ERR_INVALID_ARGUMENT, "position dtype differs from the plan's");
    total += parts[b].n;
  }
  if (pl.staged.size() >= 2)
    cmh::fail(CMH_ERR_INVALID_ARGUMENT, "two runs are staged already");
  if (total == 0) return;
  std::vector<cmh_particles> v(parts, parts + nbox);
  if (pl.input_buffers == 1) {
    // one buffer: copied now if it holds nothing that a later run needs,
    // else behind the next run's reads of it
    if (pl.staged.empty()) {
      pl.stage_inputs(parts, nbox, static_cast<cudaStream_t>(stream), 0);
      pl.staged.push_back(cmh::Plan::Staged{v, 0, false});
    } else {
      pl.staged.push_back(cmh::Plan::Staged{v, 0, true});
    }
    return;
  }
  // the buffer that neither the last run nor the newest staged inputs hold
  const int b = pl.stage_inputs(parts, nbox, static_cast<cudaStream_t>(stream),
                                1 - (pl.staged.empty() ? pl.last_buf : pl.staged.back().buf));
  pl.staged.push_back(cmh::Plan::Staged{v, b, false});
}
}  // namespace

cmh_status cmh_plan_prefetch(cmh_plan *plan, const cmh_particles *parts, void *stream) {
  CMH_API_BEGIN
  if (!plan || !parts) cmh::fail(CMH_ERR_INVALID_ARGUMENT, "plan and particles are required");
  prefetch_on(*static_cast<Plan *>(plan), parts, 1, stream);
  CMH_API_END
}

cmh_status cmh_plan_set_input_buffers(cmh_plan *plan, int32_t n) {
  CMH_API_BEGIN
  if (!plan || (n != 1 && n != 2))
    cmh::fail(CMH_ERR_INVALID_ARGUMENT, "a plan and 1 or 2 input buffers are required");
  Plan &pl = *static_cast<Plan *>(plan);
  CMH_CUDA(cudaSetDevice(pl.device));
  if (pl.side_stream) CMH_CUDA(cudaStreamSynchronize(pl.side_stream));
  pl.staged.clear();  // staged copies are dropped
  pl.input_buffers = n;
  pl.last_buf = 0;
  if (n == 1) {
    pl.in_pos[1].release();
    pl.in_vel[1].release();
  }
  CMH_API_END
}

cmh_status cmh_plan_prefetch_batch(cmh_plan *plan, const cmh_particles *parts, int32_t nbox,
                                   void *stream) {
  CMH_API_BEGIN
  if (!plan || !parts || nbox < 1)
    cmh::fail(CMH_ERR_INVALID_ARGUMENT, "plan and particles are required");
  prefetch_on(*static_cast<Plan *>(plan), parts, nbox, stream);
  CMH_API_END
}

void cmh_plan_destroy(cmh_plan *plan) { delete static_cast<Plan *>(plan); }

void cmh_catalog_free(cmh_catalog *cat) {
  if (!cat) return;
  auto *st = static_cast<cmh::CatalogStore *>(cat->impl);
  if (st && st->host_owned) {
    free(cat->props);
    free(cat->head);
    free(cat->member);
    free(cat->member_proc);
    free(cat->member_pos);
  }
  delete st;
  cat->props = nullptr;
  cat->head = nullptr;
  cat->member = nullptr;
  cat->member_proc = nullptr;
  cat->member_pos = nullptr;
  cat->impl = nullptr;
  cat->nhalos = 0;
}

namespace {

// One-shot run of cmh_fof_run / cmh_fof_run_sampled.
void fof_once(const cmh_fof_params *params, const cmh_particles *parts,
              const cmh_sampling *sampling, cmh_catalog *cat, int32_t want_member,
              cmh_sample *sample, void *stream) {
  if (!params || !cat) cmh::fail(CMH_ERR_INVALID_ARGUMENT, "params and catalog are required");
  check_parts(parts);
  memset(cat, 0, sizeof *cat);
  if (sampling) {
    if (!sample) cmh::fail(CMH_ERR_INVALID_ARGUMENT, "a sample needs its output");
    memset(sample, 0, sizeof *sample);
    if (!(sampling->samp_in >= 0.0 && sampling->samp_in <= 1.0) ||
        !(sampling->samp_out >= 0.0 && sampling->samp_out <= 1.0))
      cmh::fail(CMH_ERR_INVALID_ARGUMENT, "sampling rates must lie in [0, 1]");
  }
  const int dev = current_device();
  std::unique_ptr<Plan> pl(new Plan(*params, parts->pos_dtype, dev));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cmh_particles dp = *parts;
  // device copies of host inputs, freed on every way out
  struct Copies {
    cmh::DevBuf pos, vel, ids;
    ~Copies() {
      pos.release();
      vel.release();
      ids.release();
    }
  } cp;
  cmh::DevBuf &dpos = cp.pos, &dvel = cp.vel, &dids = cp.ids;
  if (parts->location == CMH_HOST && parts->n > 0) {
    const size_t pb = (size_t)parts->n * 3 * (parts->pos_dtype == CMH_FLOAT64 ? 8 : 4);
    const size_t vb = (size_t)parts->n * 3 * (parts->vel_dtype == CMH_FLOAT64 ? 8 : 4);
    dpos.ensure(pb);
    dvel.ensure(vb);
    CMH_CUDA(cudaMemcpyAsync(dpos.p, parts->pos, pb, cudaMemcpyHostToDevice, s));
    CMH_CUDA(cudaMemcpyAsync(dvel.p, parts->vel, vb, cudaMemcpyHostToDevice, s));
    dp.pos = dpos.p;
    dp.vel = dvel.p;
    dp.location = CMH_DEVICE;
  }
  if (sampling) {
    pl->sampling = true;
    pl->samp_in = sampling->samp_in;
    pl->samp_out = sampling->samp_out;
    pl->samp_seed = (uint64_t)(int64_t)sampling->seed;
    for (int a = 0; a < 3; a++) pl->samp_closed |= (sampling->closed_hi[a] ? 1 : 0) << a;
    pl->use_graph = false;  // one run: nothing to replay
    if (parts->id && parts->n > 0) {
      if (parts->location == CMH_HOST) {
        dids.ensure((size_t)parts->n * 8);
        CMH_CUDA(cudaMemcpyAsync(dids.p, parts->id, (size_t)parts->n * 8,
                                 cudaMemcpyHostToDevice, s));
        pl->samp_ids = dids.as<uint64_t>();
      } else {
        pl->samp_ids = parts->id;
      }
    }
  }
  pl->run(dp, want_member != 0, s);
  catalog_to_host(*pl, cat, want_member != 0, 0, s);
  if (sampling) {
    const int64_t n = parts->n;
    std::vector<uint8_t> flag((size_t)std::max<int64_t>(n, 1), 0);
    if (n > 0) {
      CMH_CUDA(cudaMemcpyAsync(flag.data(), pl->b_samp.p, (size_t)n, cudaMemcpyDeviceToHost, s));
      CMH_CUDA(cudaStreamSynchronize(s));
    }
    int64_t nin = 0, nout = 0;
    for (int64_t i = 0; i < n; i++) {
      nin += flag[i] == 1;
      nout += flag[i] == 2;
    }
    sample->inhalo = (int64_t *)malloc(sizeof(int64_t) * (size_t)std::max<int64_t>(nin, 1));
    sample->outhalo = (int64_t *)malloc(sizeof(int64_t) * (size_t)std::max<int64_t>(nout, 1));
    if (!sample->inhalo || !sample->outhalo) {
      free(sample->inhalo);
      free(sample->outhalo);
      sample->inhalo = sample->outhalo = nullptr;
      cmh::fail(CMH_ERR_OUT_OF_MEMORY, "host sample allocation failed");
    }
    for (int64_t i = 0; i < n; i++) {
      if (flag[i] == 1) sample->inhalo[sample->n_inhalo++] = i;
      else if (flag[i] == 2) sample->outhalo[sample->n_outhalo++] = i;
    }
  }
}

}  // namespace

cmh_status cmh_fof_run(const cmh_fof_params *params, const cmh_particles *parts,
                       cmh_catalog *cat, int32_t want_member, void *stream) {
  CMH_API_BEGIN
  fof_once(params, parts, nullptr, cat, want_member, nullptr, stream);
  CMH_API_END
}

cmh_status cmh_fof_run_sampled(const cmh_fof_params *params, const cmh_particles *parts,
                               const cmh_sampling *sampling, cmh_catalog *cat,
                               int32_t want_member, cmh_sample *sample, void *stream) {
  CMH_API_BEGIN
  if (!sampling) cmh::fail(CMH_ERR_INVALID_ARGUMENT, "sampling parameters are required");
  fof_once(params, parts, sampling, cat, want_member, sample, stream);
  CMH_API_END
}

void cmh_sample_free(cmh_sample *sample) {
  if (!sample) return;
  free(sample->inhalo);
  free(sample->outhalo);
  memset(sample, 0, sizeof *sample);
}

namespace {
std::vector<cmh::BoxSpec> make_specs(Plan &pl, const cmh_fof_params *params,
                                     const cmh_particles *parts, int32_t nbox) {
  std::vector<cmh::BoxSpec> specs(nbox);
  for (int b = 0; b < nbox; b++) {
    check_parts(&parts[b]);
    if (parts[b].location != CMH_DEVICE)
      cmh::fail(CMH_ERR_INVALID_ARGUMENT, "batched runs take device-resident particles");
    if (parts[b].pos_dtype != pl.pos_dtype)
      cmh::fail(CMH_ERR_INVALID_ARGUMENT, "all boxes of a batch share the position dtype");
    if (params[b].precision != params[0].precision)
      cmh::fail(CMH_ERR_INVALID_ARGUMENT, "all boxes of a batch share the precision mode");
    cmh::BoxSpec &sp = specs[b];
    sp.params = params[b];
    if (params[b].varlink) {
      if (params[b].ltab_n < 2 || !params[b].ltab)
        cmh::fail(CMH_ERR_INVALID_ARGUMENT, "variable linking length needs a table");
      sp.ltab.assign(params[b].ltab, params[b].ltab + params[b].ltab_n);
    }
    sp.params.ltab = nullptr;
    sp.pos = parts[b].pos;
    sp.vel = parts[b].vel;
    sp.vel_f64 = parts[b].vel_dtype == CMH_FLOAT64;
    sp.n = parts[b].n;
  }
  pl.fp32 = params[0].precision == CMH_FP32_RECHECK;
  return specs;
}

// Host-resident boxes (all of a batch, or none) are copied into the plan's
// input buffers first, or taken from a prefetch of the same boxes.
void run_batch_on(Plan &pl, const cmh_fof_params *params, const cmh_particles *parts,
                  int32_t nbox, cmh_catalog *cats, cudaStream_t s) {
  int host = 0;
  int64_t total = 0;
  for (int b = 0; b < nbox; b++) {
    check_parts(&parts[b]);
    host += parts[b].location == CMH_HOST;
    total += parts[b].n;
  }
  if (host != 0 && host != nbox)
    cmh::fail(CMH_ERR_INVALID_ARGUMENT,
              "a batch's boxes are all host-resident or all device-resident");
  std::vector<cmh_particles> dp;
  if (host) {
    for (int b = 0; b < nbox; b++)
      if (parts[b].pos_dtype != pl.pos_dtype)
        cmh::fail(CMH_ERR_INVALID_ARGUMENT, "all boxes of a batch share the position dtype");
    if (total > 0) {
      dp = pl.take_inputs(parts, nbox, s);
    } else {
      dp.assign(parts, parts + nbox);
      for (cmh_particles &q : dp) q.location = CMH_DEVICE;  // nothing to read
    }
    parts = dp.data();
  }
  struct Reset {
    Plan &p;
    ~Reset() { p.vel_wait = false; }
  } reset{pl};
  pl.run_batch(make_specs(pl, params, parts, nbox), false, s);
  for (int b = 0; b < nbox; b++) catalog_to_host(pl, &cats[b], false, b, s);
}
}  // namespace

cmh_status cmh_plan_autotune(cmh_plan *plan, const cmh_fof_params *params,
                             const cmh_particles *parts, int32_t nbox, int32_t repeats,
                             void *stream, cmh_tuning *out) {
  CMH_API_BEGIN
  if (!plan || !params || !parts || nbox < 1)
    cmh::fail(CMH_ERR_INVALID_ARGUMENT, "plan, params and particles are required");
  Plan &pl = *static_cast<Plan *>(plan);
  cmh_tuning t = pl.autotune(make_specs(pl, params, parts, nbox), repeats,
                             static_cast<cudaStream_t>(stream));
  if (out) *out = t;
  CMH_API_END
}

cmh_status cmh_plan_set_tuning(cmh_plan *plan, const cmh_tuning *tuning) {
  CMH_API_BEGIN
  if (!plan || !tuning) cmh::fail(CMH_ERR_INVALID_ARGUMENT, "plan and tuning are required");
  if (!(tuning->cell_scale > 0) || tuning->cell_scale > 64 || tuning->dense_min < 1)
    cmh::fail(CMH_ERR_INVALID_ARGUMENT, "cell_scale must be in (0, 64] and dense_min >= 1");
  Plan &pl = *static_cast<Plan *>(plan);
  pl.cell_scale = tuning->cell_scale;
  pl.dense_min = (uint32_t)tuning->dense_min;
  CMH_API_END
}

cmh_status cmh_fof_run_batch(const cmh_fof_params *params, const cmh_particles *parts,
                             int32_t nbox, cmh_catalog *cats, void *stream) {
  CMH_API_BEGIN
  if (!params || !parts || !cats || nbox < 0)
    cmh::fail(CMH_ERR_INVALID_ARGUMENT, "params, particles and catalogs are required");
  for (int b = 0; b < nbox; b++) memset(&cats[b], 0, sizeof cats[b]);
  if (nbox == 0) return CMH_OK;
  const int dev = current_device();
  std::unique_ptr<Plan> pl(new Plan(params[0], parts[0].pos_dtype, dev));
  pl->use_graph = false;
  run_batch_on(*pl, params, parts, nbox, cats, static_cast<cudaStream_t>(stream));
  CMH_API_END
}

cmh_status cmh_plan_run_batch(cmh_plan *plan, const cmh_fof_params *params,
                              const cmh_particles *parts, int32_t nbox, cmh_catalog *cats,
                              void *stream) {
  CMH_API_BEGIN
  if (!plan || !params || !parts || !cats || nbox < 1)
    cmh::fail(CMH_ERR_INVALID_ARGUMENT, "plan, params, particles and catalogs are required");
  for (int b = 0; b < nbox; b++) memset(&cats[b], 0, sizeof cats[b]);
  run_batch_on(*static_cast<Plan *>(plan), params, parts, nbox, cats,
               static_cast<cudaStream_t>(stream));
  CMH_API_END
}

cmh_status cmh_plan_run_batch_status(cmh_plan *plan, const cmh_fof_params *params,
                                     const cmh_particles *parts, int32_t nbox,
                                     cmh_catalog *cats, cmh_status *box_status, void *stream) {
  CMH_API_BEGIN
  if (!plan || !params || !parts || !cats || !box_status || nbox < 1)
    cmh::fail(CMH_ERR_INVALID_ARGUMENT,
              "plan, params, particles, catalogs and statuses are required");
  Plan &pl = *static_cast<Plan *>(plan);
  // each box on its own: its particle description, then its geometry
  std::vector<int> ok;
  int precision = -1;
  for (int b = 0; b < nbox; b++) {
    memset(&cats[b], 0, sizeof cats[b]);
    box_status[b] = CMH_OK;
    try {
      check_parts(&parts[b]);
      if (parts[b].location != parts[0].location)
        cmh::fail(CMH_ERR_INVALID_ARGUMENT,
                  "a batch's boxes are all host-resident or all device-resident");
      if (parts[b].pos_dtype != pl.pos_dtype)
        cmh::fail(CMH_ERR_INVALID_ARGUMENT, "position dtype differs from the plan's");
      const cmh_fof_params &p = params[b];
      if (!(p.linklength > 0) || !(p.boundary >= 0) ||
          (p.precision != CMH_PLAIN_FP64 && p.precision != CMH_FP32_RECHECK))
        cmh::fail(CMH_ERR_INVALID_ARGUMENT, "bad Linklength, Boundarysize or precision");
      if (precision >= 0 && p.precision != precision)
        cmh::fail(CMH_ERR_INVALID_ARGUMENT, "all boxes of a batch share the precision mode");
      std::vector<double> ltab;
      if (p.varlink) {
        if (p.ltab_n < 2 || !p.ltab)
          cmh::fail(CMH_ERR_INVALID_ARGUMENT, "variable linking length needs a table");
        ltab.assign(p.ltab, p.ltab + p.ltab_n);
      }
      (void)pl.make_geometry(p, ltab, parts[b].n, 0);
      precision = p.precision;
      ok.push_back(b);
    } catch (const Error &e) {
      box_status[b] = e.code;
    }
  }
  if (ok.empty()) return CMH_OK;
  std::vector<cmh_fof_params> sp;
  std::vector<cmh_particles> sq;
  std::vector<cmh_catalog> sc(ok.size());
  for (int b : ok) {
    sp.push_back(params[b]);
    sq.push_back(parts[b]);
  }
  try {
    run_batch_on(pl, sp.data(), sq.data(), (int32_t)ok.size(), sc.data(),
                 static_cast<cudaStream_t>(stream));
  } catch (const Error &e) {
    for (cmh_catalog &c : sc) cmh_catalog_free(&c);
    for (int b : ok) box_status[b] = e.code;
    throw;
  }
  for (size_t i = 0; i < ok.size(); i++) cats[ok[i]] = sc[i];
  CMH_API_END
}

cmh_status cmh_plan_set_limits(cmh_plan *plan, const cmh_limits *limits) {
  CMH_API_BEGIN
  if (!plan || !limits) cmh::fail(CMH_ERR_INVALID_ARGUMENT, "plan and limits are required");
  auto pick = [](int64_t v, uint32_t def) -> uint32_t {
    if (v < 0) return def;
    if (v > 0x7fffffffll) cmh::fail(CMH_ERR_INVALID_ARGUMENT, "limits must be below 2^31");
    return (uint32_t)v;
  };
  const uint32_t u = pick(limits->union_attempts, cmh::kUnionCap);
  const uint32_t w = pick(limits->lookback_polls, cmh::kSpinCap);
  Plan &pl = *static_cast<Plan *>(plan);
  pl.union_cap = u;
  pl.spin_cap = w;
  CMH_API_END
}

cmh_status cmh_plan_set_graph(cmh_plan *plan, int32_t enable) {
  CMH_API_BEGIN
  if (!plan) cmh::fail(CMH_ERR_INVALID_ARGUMENT, "plan is required");
  static_cast<Plan *>(plan)->use_graph = enable != 0;
  CMH_API_END
}

}  // extern "C"
