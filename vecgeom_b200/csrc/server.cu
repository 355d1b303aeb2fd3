// server.cu -- continuous batching of navigation requests (vgb_server_*).
//
// Device memory holds a fixed table of track slots, carved into chunks of
// kChunk tracks.  A request owns whole chunks; the last one is padded with
// finished tracks.  Every iteration (vgb_server_step):
//   1. admit: queued requests, in arrival order, take free chunks; a request
//      that does not fit is passed over by later ones that do (a large request
//      does not hold up the small ones behind it), until it has been passed
//      over kMaxBypass times, after which nothing more is admitted ahead of it;
//      the points of all admitted requests go to the device in one copy from a
//      pinned staging buffer, and one launch scatters them into their slots,
//      locates them (LocatePoint from the world) and clears their counters;
//   2. step: one launch over the chunks of all admitted requests advances every
//      live track by up to steps_per_launch steps, each GetSafety and
//      FindNextBoundaryAndStep (one warp per track, the navigator of
//      navigation.cuh), and counts the tracks still live per chunk;
//   3. retire: the requests whose chunks have no live track are finished; one
//      launch gathers their results into a staging buffer, one copy brings them
//      to pinned host memory, and their chunks are free for the next admission.
// Requests that arrive while others are in flight join at the next iteration,
// so their steps share launches with the older requests' steps.
#include <algorithm>
#include <cstring>
#include <deque>
#include <map>
#include <vector>

#include "navigation.cuh"

using namespace vgb;

namespace vgb {
namespace {

constexpr int kChunk = 256;
constexpr int kSrvBlock = 128;
constexpr int kSrvWarps = kSrvBlock / 32;
constexpr uint64_t kFnvOffset = 0xcbf29ce484222325ull;
constexpr uint64_t kFnvPrime = 0x100000001b3ull;

struct Slots {
  double *x, *y, *z, *dx, *dy, *dz;
  unsigned char *states;
  int64_t stride;
  int32_t *nsteps;
  uint64_t *hash;
  uint8_t *done;
};

// Per-track record of a finished request, as staged for the copy to the host.
struct TrackResult {
  double x, y, z;
  uint64_t hash;
  int32_t nsteps;
  int32_t pad;
};

VGB_HD uint64_t fnv_bytes(uint64_t h, const void *p, int n) {
  const unsigned char *b = static_cast<const unsigned char *>(p);
  for (int i = 0; i < n; ++i) {
    h ^= b[i];
    h *= kFnvPrime;
  }
  return h;
}

// slot of the t-th track of the chunk list
VGB_D int64_t slot_of(const int32_t *chunks, int64_t t) {
  return (int64_t)chunks[t / kChunk] * kChunk + (t % kChunk);
}

// in: 6 arrays of ntracks (x, y, z, dx, dy, dz) in chunk-list order; valid[t]
// marks the request's tracks (the rest pad the last chunk of each request)
template <uint32_t kMask>
__global__ void __launch_bounds__(kSrvBlock)
    k_srv_admit(const NavGeom G, const int32_t *chunks, int64_t ntracks, const double *in,
                const uint8_t *valid, Slots S, uint32_t *flags) {
  using Nav = Navigator<WarpLanes, kMask>;
  const int64_t warps = (int64_t)gridDim.x * kSrvWarps;
  for (int64_t t = (int64_t)blockIdx.x * kSrvWarps + threadIdx.x / 32; t < ntracks; t += warps) {
    const int64_t s = slot_of(chunks, t);
    const bool v = valid[t] != 0;
    NavPath p;
    bool ok = true;
    V3<double> x = {0., 0., 0.};
    if (v) {
      x = {in[t], in[ntracks + t], in[2 * ntracks + t]};
      ok = Nav::locate_from_world(G, p, x);
    } else {
      p.level = 0;
      p.boundary = false;
    }
    if (WarpLanes::lane() == 0) {
      if (!ok) {
        atomicOr(flags, (uint32_t)VGB_NAV_ERR_DEPTH);
        p.level = 0;
      }
      nav_store(p, NavStateRef{S.states + s * S.stride}, G.max_depth);
      S.x[s] = x.x;
      S.y[s] = x.y;
      S.z[s] = x.z;
      S.dx[s] = v ? in[3 * ntracks + t] : 0.;
      S.dy[s] = v ? in[4 * ntracks + t] : 0.;
      S.dz[s] = v ? in[5 * ntracks + t] : 0.;
      S.nsteps[s] = 0;
      S.hash[s] = kFnvOffset;
      S.done[s] = (v && p.level > 0) ? 0 : 1;
    }
  }
}

template <uint32_t kMask, bool kScreen>
__global__ void __launch_bounds__(kSrvBlock)
    k_srv_step(const NavGeom G, const int32_t *chunks, int64_t ntracks, Slots S, double pstep,
               int32_t max_steps, int32_t steps_per_launch, int32_t *live, uint32_t *flags) {
  using Nav = Navigator<WarpLanes, kMask, kScreen>;
  const int64_t warps = (int64_t)gridDim.x * kSrvWarps;
  const bool lane0 = WarpLanes::lane() == 0;
  for (int64_t t = (int64_t)blockIdx.x * kSrvWarps + threadIdx.x / 32; t < ntracks; t += warps) {
    const int64_t s = slot_of(chunks, t);
    if (S.done[s]) continue;
    NavPath cur, nxt;
    nav_load(cur, NavStateRef{S.states + s * S.stride});
    V3<double> p = {S.x[s], S.y[s], S.z[s]};
    const V3<double> d = {S.dx[s], S.dy[s], S.dz[s]};
    int32_t k = S.nsteps[s];
    uint64_t h = S.hash[s];
    bool ok = true;
    for (int it = 0; it < steps_per_launch && cur.level > 0 && k < max_steps; ++it) {
      const DXform m = nav_top_matrix(G, cur);
      const V3<double> lp = xf_point(m, p);
      const V3<double> ld = xf_dir(m, d);
      const double sf = Nav::safety(G, cur, lp);
      double st = 0.;
      ok = Nav::step(G, cur, nxt, lp, ld, pstep, st);
      if (!ok) break;
      const int32_t id = nxt.top();
      h = fnv_bytes(h, &id, 4);
      h = fnv_bytes(h, &st, 8);
      h = fnv_bytes(h, &sf, 8);
      p = {p.x + d.x * st, p.y + d.y * st, p.z + d.z * st};
      cur = nxt;
      ++k;
    }
    if (lane0) {
      const bool fin = !ok || cur.level == 0 || k >= max_steps;
      if (!ok) atomicOr(flags, (uint32_t)VGB_NAV_ERR_DEPTH);
      nav_store(cur, NavStateRef{S.states + s * S.stride}, G.max_depth);
      S.x[s] = p.x;
      S.y[s] = p.y;
      S.z[s] = p.z;
      S.nsteps[s] = ok ? k : -1;
      S.hash[s] = h;
      S.done[s] = fin ? 1 : 0;
      if (!fin) atomicAdd(live + t / kChunk, 1);
    }
  }
}

// results of the listed chunks' slots, in chunk-list order
__global__ void k_srv_gather(const int32_t *chunks, int64_t ntracks, Slots S, TrackResult *out) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntracks;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = slot_of(chunks, t);
    out[t] = TrackResult{S.x[s], S.y[s], S.z[s], S.hash[s], S.nsteps[s], 0};
  }
}

NavGeom server_geom(const vgb_geometry *g) {
  NavGeom G;
  G.params = g->dev.params;
  G.unplaced = g->dev.unplaced;
  G.placed = g->dev.placed;
  G.xforms = g->dev.xforms;
  G.raw = g->dev.raw;
  G.logicals = g->dev.logicals;
  G.daughters = g->dev.daughters;
  G.pl_box = g->dev.pl_box;
  G.ab_box = g->dev.ab_box;
  G.ab_slot = g->dev.ab_slot;
  G.world = g->world;
  G.max_depth = g->max_depth;
  return G;
}

int srv_grid(int64_t ntracks) {
  const int64_t want = (ntracks + kSrvWarps - 1) / kSrvWarps;
  const int64_t cap = 148 * 16;
  return (int)std::max<int64_t>(1, std::min(want, cap));
}

struct Request {
  int64_t id = -1;
  int64_t n = 0;
  int32_t bypassed = 0;    // admissions of later requests while this one waited
  std::vector<double> in;  // x, y, z, dx, dy, dz (6 n)
  std::vector<int32_t> chunks;
  std::vector<TrackResult> out;
};

}  // namespace
}  // namespace vgb

struct vgb_server {
  const vgb_geometry *g = nullptr;
  int device = -1;
  int32_t steps_per_launch = 8;
  int32_t max_steps = 1000;
  double pstep = 1e30;
  int64_t nchunks = 0;
  int64_t bytes = 0;
  vgb::Slots S{};
  int32_t *d_chunks = nullptr;   // chunk list of the current launch
  int32_t *d_live = nullptr;     // live tracks per listed chunk
  double *d_in = nullptr;        // staged inputs of an admission (6 * slots)
  uint8_t *d_valid = nullptr;    // request track or padding, per staged track
  vgb::TrackResult *d_out = nullptr;  // gathered results of a retirement
  double *h_in = nullptr;        // pinned host mirrors of the three buffers
  uint8_t *h_valid = nullptr;
  vgb::TrackResult *h_out = nullptr;
  int32_t *h_chunks = nullptr;   // chunk lists of the step and retire launches
  int32_t *h_achunks = nullptr;  // chunk list of the admit launch (copied asynchronously)
  int32_t *h_live = nullptr;
  cudaStream_t stream = nullptr;
  std::vector<int32_t> free_chunks;
  std::deque<vgb::Request *> queue;
  std::vector<vgb::Request *> active;
  std::map<int64_t, vgb::Request *> done;
  int64_t next_id = 0;
  bool all_shapes = false;
  bool screen = false;  // FP32+refine: float screen on the daughter loops
};

namespace vgb {
namespace {

template <class T> cudaError_t srv_alloc(vgb_server *s, T **p, size_t n) {
  cudaError_t e = cudaMalloc((void **)p, std::max<size_t>(1, n) * sizeof(T));
  if (e == cudaSuccess) s->bytes += (int64_t)(std::max<size_t>(1, n) * sizeof(T));
  return e;
}
template <class T> cudaError_t srv_pin(T **p, size_t n) {
  return cudaHostAlloc((void **)p, std::max<size_t>(1, n) * sizeof(T), cudaHostAllocDefault);
}

void srv_free(vgb_server *s) {
  Slots &S = s->S;
  void *ptrs[] = {S.x,         S.y,         S.z,      S.dx,       S.dy,    S.dz,
                  S.states,    S.nsteps,    S.hash,   S.done,     s->d_chunks,
                  s->d_live,   s->d_in,     s->d_valid, s->d_out};
  for (void *p : ptrs) cudaFree(p);
  void *pins[] = {s->h_in, s->h_valid, s->h_out, s->h_chunks, s->h_achunks, s->h_live};
  for (void *p : pins) cudaFreeHost(p);
  if (s->stream) cudaStreamDestroy(s->stream);
  for (Request *r : s->queue) delete r;
  for (Request *r : s->active) delete r;
  for (auto &kv : s->done) delete kv.second;
}

template <uint32_t kMask> void launch_admit(vgb_server *s, int64_t nt) {
  k_srv_admit<kMask><<<srv_grid(nt), kSrvBlock, 0, s->stream>>>(
      server_geom(s->g), s->d_chunks, nt, s->d_in, s->d_valid, s->S, s->g->dev.nav_flags);
}
template <uint32_t kMask> void launch_step(vgb_server *s, int64_t nt) {
  if (s->screen)
    k_srv_step<kMask, true><<<srv_grid(nt), kSrvBlock, 0, s->stream>>>(
        server_geom(s->g), s->d_chunks, nt, s->S, s->pstep, s->max_steps, s->steps_per_launch,
        s->d_live, s->g->dev.nav_flags);
  else
    k_srv_step<kMask, false><<<srv_grid(nt), kSrvBlock, 0, s->stream>>>(
        server_geom(s->g), s->d_chunks, nt, s->S, s->pstep, s->max_steps, s->steps_per_launch,
        s->d_live, s->g->dev.nav_flags);
}

// A waiting request is passed over by at most this many later admissions; then
// the later requests wait behind it until the slots it needs are free.
constexpr int32_t kMaxBypass = 16;

// Admits queued requests while free chunks last, all in one copy and one
// launch: in arrival order, each request that fits; one that does not stays
// queued and later ones may pass it, up to kMaxBypass times.
vgb_status admit(vgb_server *s) {
  std::vector<Request *> batch;
  int64_t nc = 0;
  std::vector<Request *> waiting;  // passed over in this admission, in order
  while (!s->queue.empty()) {
    Request *r = s->queue.front();
    const int64_t need = (r->n + kChunk - 1) / kChunk;
    if (need > (int64_t)s->free_chunks.size()) {
      if (r->bypassed >= kMaxBypass) break;  // it goes next: nothing passes it
      s->queue.pop_front();
      waiting.push_back(r);
      continue;
    }
    s->queue.pop_front();
    for (Request *w : waiting) ++w->bypassed;
    r->chunks.assign(s->free_chunks.end() - need, s->free_chunks.end());
    s->free_chunks.resize(s->free_chunks.size() - need);
    batch.push_back(r);
    nc += need;
  }
  // the passed-over requests go back to the front, in their arrival order
  for (auto it = waiting.rbegin(); it != waiting.rend(); ++it) s->queue.push_front(*it);
  if (batch.empty()) return VGB_OK;
  const int64_t nt = nc * kChunk;
  int64_t c = 0;
  for (Request *r : batch) {
    for (size_t k = 0; k < r->chunks.size(); ++k, ++c) {
      s->h_achunks[c] = r->chunks[k];
      for (int j = 0; j < kChunk; ++j) {
        const int64_t src = (int64_t)k * kChunk + j, dst = c * kChunk + j;
        const bool v = src < r->n;
        s->h_valid[dst] = v ? 1 : 0;
        for (int a = 0; a < 6; ++a) s->h_in[a * nt + dst] = v ? r->in[a * r->n + src] : 0.;
      }
    }
    std::vector<double>().swap(r->in);
    s->active.push_back(r);
  }
  cudaError_t e = cudaMemcpyAsync(s->d_in, s->h_in, 6 * nt * sizeof(double),
                                  cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(s->d_valid, s->h_valid, nt, cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(s->d_chunks, s->h_achunks, nc * sizeof(int32_t), cudaMemcpyHostToDevice,
                        s->stream);
  if (e != cudaSuccess) return cuda_error(e, "vgb_server_step: admit copy");
  if (s->all_shapes)
    launch_admit<kNavMaskAll>(s, nt);
  else
    launch_admit<kNavMaskBoxTubeTrd>(s, nt);
  count_launch();
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_error(e, "vgb_server_step: admit");
  return VGB_OK;
}

}  // namespace
}  // namespace vgb

extern "C" {

vgb_status vgb_server_create(const vgb_geometry *g, int64_t max_tracks, int32_t steps_per_launch,
                             int32_t max_steps, double pstep, int32_t precision,
                             vgb_server **server) {
  if (!server) return set_error(VGB_EINVAL, "vgb_server_create: server is NULL");
  *server = nullptr;
  if (precision != VGB_PREC_FP64 && precision != VGB_PREC_FP32_REFINE)
    return set_error(VGB_EINVAL, "vgb_server_create: unknown precision %d", precision);
  if (!g || !g->closed || g->world < 0)
    return set_error(VGB_EINVAL, "vgb_server_create: geometry not closed or without world");
  if (g->max_depth > kNavMaxLevels)
    return set_error(VGB_ENOTSUP, "vgb_server_create: geometry deeper than %d levels",
                     kNavMaxLevels);
  if (max_tracks < 0 || steps_per_launch < 1 || max_steps < 0)
    return set_error(VGB_EINVAL, "vgb_server_create: bad capacity or step counts");
  const int64_t stride = nav_state_stride(g->max_depth);
  // slots (points, state, counters) + staged inputs + gathered results
  const int64_t per_track = 6 * 8 + stride + 4 + 8 + 1 + 6 * 8 + 1 + (int64_t)sizeof(TrackResult);
  size_t fr = 0, tot = 0;
  cudaError_t e = cudaMemGetInfo(&fr, &tot);
  if (e != cudaSuccess) return cuda_error(e, "vgb_server_create: cudaMemGetInfo");
  if (max_tracks == 0) max_tracks = std::min<int64_t>((int64_t)(fr / 4) / per_track, (int64_t)1 << 22);
  const int64_t nchunks = (max_tracks + kChunk - 1) / kChunk;
  const int64_t nslots = nchunks * kChunk;
  if ((double)nslots * per_track > 0.9 * (double)fr)
    return set_error(VGB_ENOMEM, "vgb_server_create: %lld track slots need %lld bytes, %zu free",
                     (long long)nslots, (long long)(nslots * per_track), fr);
  vgb_server *s = new vgb_server;
  s->g = g;
  s->device = g->device;
  s->steps_per_launch = steps_per_launch;
  s->max_steps = max_steps;
  s->pstep = pstep;
  s->nchunks = nchunks;
  s->all_shapes = (g->type_mask & ~kNavMaskBoxTubeTrd) != 0;
  s->screen = precision == VGB_PREC_FP32_REFINE;
  Slots &S = s->S;
  S.stride = stride;
  e = cudaSuccess;
  double **coords[] = {&S.x, &S.y, &S.z, &S.dx, &S.dy, &S.dz};
  for (double **c : coords)
    if (e == cudaSuccess) e = srv_alloc(s, c, nslots);
  if (e == cudaSuccess) e = srv_alloc(s, &S.states, nslots * stride);
  if (e == cudaSuccess) e = srv_alloc(s, &S.nsteps, nslots);
  if (e == cudaSuccess) e = srv_alloc(s, &S.hash, nslots);
  if (e == cudaSuccess) e = srv_alloc(s, &S.done, nslots);
  if (e == cudaSuccess) e = srv_alloc(s, &s->d_chunks, nchunks);
  if (e == cudaSuccess) e = srv_alloc(s, &s->d_live, nchunks);
  if (e == cudaSuccess) e = srv_alloc(s, &s->d_in, 6 * nslots);
  if (e == cudaSuccess) e = srv_alloc(s, &s->d_valid, nslots);
  if (e == cudaSuccess) e = srv_alloc(s, &s->d_out, nslots);
  if (e == cudaSuccess) e = srv_pin(&s->h_in, 6 * nslots);
  if (e == cudaSuccess) e = srv_pin(&s->h_valid, nslots);
  if (e == cudaSuccess) e = srv_pin(&s->h_out, nslots);
  if (e == cudaSuccess) e = srv_pin(&s->h_chunks, nchunks);
  if (e == cudaSuccess) e = srv_pin(&s->h_achunks, nchunks);
  if (e == cudaSuccess) e = srv_pin(&s->h_live, nchunks);
  if (e == cudaSuccess) e = cudaMemset(S.done, 1, nslots);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    srv_free(s);
    delete s;
    return cuda_error(e, "vgb_server_create");
  }
  s->free_chunks.resize(nchunks);
  for (int64_t c = 0; c < nchunks; ++c) s->free_chunks[c] = (int32_t)(nchunks - 1 - c);
  *server = s;
  return VGB_OK;
}

vgb_status vgb_server_destroy(vgb_server *s) {
  if (!s) return VGB_OK;
  cudaStreamSynchronize(s->stream);
  srv_free(s);
  delete s;
  return VGB_OK;
}

vgb_status vgb_server_info(const vgb_server *s, int64_t *max_tracks, int64_t *device_bytes) {
  if (!s) return set_error(VGB_EINVAL, "vgb_server_info: server is NULL");
  if (max_tracks) *max_tracks = s->nchunks * kChunk;
  if (device_bytes) *device_bytes = s->bytes;
  return VGB_OK;
}

vgb_status vgb_server_submit(vgb_server *s, int64_t n, const double *x, const double *y,
                             const double *z, const double *dx, const double *dy,
                             const double *dz, int64_t *request_id) {
  if (!s) return set_error(VGB_EINVAL, "vgb_server_submit: server is NULL");
  if (n < 0 || (n > 0 && (!x || !y || !z || !dx || !dy || !dz)))
    return set_error(VGB_EINVAL, "vgb_server_submit: bad track arrays");
  if ((n + kChunk - 1) / kChunk > s->nchunks)
    return set_error(VGB_ENOSPC, "vgb_server_submit: %lld tracks exceed the %lld slots",
                     (long long)n, (long long)(s->nchunks * kChunk));
  Request *r = new Request;
  r->id = s->next_id++;
  r->n = n;
  r->in.resize(6 * n);
  const double *src[6] = {x, y, z, dx, dy, dz};
  for (int k = 0; k < 6; ++k)
    if (n) std::memcpy(r->in.data() + k * n, src[k], n * sizeof(double));
  if (n == 0)
    s->done[r->id] = r;
  else
    s->queue.push_back(r);
  if (request_id) *request_id = r->id;
  return VGB_OK;
}

vgb_status vgb_server_step(vgb_server *s, int64_t *completed, int32_t max_completed,
                           int32_t *ncompleted, int64_t *live, int64_t *queued) {
  if (!s) return set_error(VGB_EINVAL, "vgb_server_step: server is NULL");
  if (ncompleted) *ncompleted = 0;
  int dev = -1;
  cudaGetDevice(&dev);
  if (dev != s->device)
    return set_error(VGB_EINVAL, "vgb_server_step: current device is not the server's");
  vgb_status st = admit(s);
  if (st != VGB_OK) return st;
  // chunk list of every admitted request
  int64_t nc = 0;
  std::vector<std::pair<int64_t, int64_t>> span(s->active.size());
  for (size_t k = 0; k < s->active.size(); ++k) {
    span[k].first = nc;
    for (int32_t c : s->active[k]->chunks) s->h_chunks[nc++] = c;
    span[k].second = nc;
  }
  int64_t live_total = 0;
  if (nc > 0) {
    cudaError_t e = cudaMemcpyAsync(s->d_chunks, s->h_chunks, nc * sizeof(int32_t),
                                    cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->d_live, 0, nc * sizeof(int32_t), s->stream);
    if (e != cudaSuccess) return cuda_error(e, "vgb_server_step: chunk list");
    const int64_t nt = nc * kChunk;
    if (s->all_shapes)
      launch_step<kNavMaskAll>(s, nt);
    else
      launch_step<kNavMaskBoxTubeTrd>(s, nt);
    count_launch();
    e = cudaGetLastError();
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(s->h_live, s->d_live, nc * sizeof(int32_t), cudaMemcpyDeviceToHost,
                          s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return cuda_error(e, "vgb_server_step: step");
  }
  // retire: gather the finished requests' results in one launch and one copy
  std::vector<Request *> still, fin;
  int64_t nf = 0;
  for (size_t k = 0; k < s->active.size(); ++k) {
    int64_t l = 0;
    for (int64_t c = span[k].first; c < span[k].second; ++c) l += s->h_live[c];
    live_total += l;
    Request *r = s->active[k];
    if (l == 0) {
      fin.push_back(r);
      nf += (int64_t)r->chunks.size();
    } else {
      still.push_back(r);
    }
  }
  if (!fin.empty()) {
    int64_t c = 0;
    for (Request *r : fin)
      for (int32_t ch : r->chunks) s->h_chunks[c++] = ch;
    const int64_t nt = nf * kChunk;
    cudaError_t e = cudaMemcpyAsync(s->d_chunks, s->h_chunks, nf * sizeof(int32_t),
                                    cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) {
      const int grid = (int)std::min<int64_t>((nt + 255) / 256, 148 * 8);
      k_srv_gather<<<grid, 256, 0, s->stream>>>(s->d_chunks, nt, s->S, s->d_out);
      count_launch();
      e = cudaGetLastError();
    }
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(s->h_out, s->d_out, nt * sizeof(TrackResult), cudaMemcpyDeviceToHost,
                          s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return cuda_error(e, "vgb_server_step: retire");
    int64_t base = 0;
    for (Request *r : fin) {
      r->out.assign(s->h_out + base, s->h_out + base + r->n);
      base += (int64_t)r->chunks.size() * kChunk;
      for (int32_t ch : r->chunks) s->free_chunks.push_back(ch);
      r->chunks.clear();
      s->done[r->id] = r;
    }
  }
  int32_t nout = 0;
  for (Request *r : fin)
    if (completed && nout < max_completed) completed[nout++] = r->id;
  s->active.swap(still);
  if (ncompleted) *ncompleted = nout;
  if (live) *live = live_total;
  if (queued) *queued = (int64_t)s->queue.size();
  return VGB_OK;
}

vgb_status vgb_server_result(vgb_server *s, int64_t request_id, int32_t *nsteps, double *x,
                             double *y, double *z, uint64_t *hash) {
  if (!s) return set_error(VGB_EINVAL, "vgb_server_result: server is NULL");
  auto it = s->done.find(request_id);
  if (it == s->done.end())
    return set_error(VGB_EINVAL, "vgb_server_result: request %lld is not finished",
                     (long long)request_id);
  Request *r = it->second;
  for (int64_t t = 0; t < r->n; ++t) {
    const TrackResult &o = r->out[t];
    if (nsteps) nsteps[t] = o.nsteps;
    if (x) x[t] = o.x;
    if (y) y[t] = o.y;
    if (z) z[t] = o.z;
    if (hash) hash[t] = o.hash;
  }
  s->done.erase(it);
  delete r;
  return VGB_OK;
}

}  // extern "C"
