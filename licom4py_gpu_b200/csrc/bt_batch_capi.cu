// bt_batch_capi.cu - C-ABI of the batched rounds (bt_batch_*, include/licom_bt.h).
//
// A batch object owns a small ring of member tables: for each call the host
// sorts the members by substep count (largest first), writes their stage
// pointers, geometry indices and prefix offsets into a pinned slot, copies it
// to the slot's device twin on the call's stream and launches the round.  A
// slot is reused only after the GPU has finished the call that last used it
// (an event per slot), so consecutive calls on any streams never overwrite a
// table that a running round still reads.

#include <algorithm>
#include <numeric>
#include <string>
#include <vector>

#include "bt_batch.cuh"
#include "bt_plan.cuh"

using namespace bt;

namespace {

int bfail(int code, const std::string& msg) { return set_error(code, msg); }
int bcuda(cudaError_t e, const char* what) { return bfail(BT_ECUDA, std::string(what) + ": " + cudaGetErrorString(e)); }

constexpr int kSlots = 4;
constexpr int kMaxGeo = 16;

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Member scratch layout: stage fields Y (3) [+ Z (3) for RK3], then the face
// cache blocks, every part 256-byte aligned.
struct ScratchLayout {
  size_t field, face, total;
  int nfields;
};
ScratchLayout scratch_layout(const bt_plan* p, int rk) {
  ScratchLayout L;
  L.field = align256(p->field_elems * p->esize());
  L.face = align256(face_cache_elems(p->n) * p->esize());
  L.nfields = rk == 3 ? 6 : 3;
  L.total = L.nfields * L.field + L.face;
  return L;
}

}  // namespace

struct bt_batch {
  int dtype = BT_F64, device = 0, max_members = 0;
  TileCfg tile{8, 32};
  int mode = BT_MODE_PERSISTENT;
  int max_ctas = 0;
  long long spin_limit = 1ll << 24;
  int last_grid = 0;
  size_t geo_bytes = 0, desc_bytes = 0, off_bytes = 0, slot_bytes = 0;
  unsigned char* d_slots = nullptr;
  unsigned char* h_slots = nullptr;
  cudaEvent_t ev[kSlots] = {};
  bool used[kSlots] = {};
  int next = 0;
  unsigned* d_flags = nullptr;  // [0] barrier counter, [1] error bits
};

namespace {

template <typename T>
int batch_round(bt_batch* b, const bt_member* mem, int count, int rk, cudaStream_t s) {
  // order: substeps descending, stable (members still running form a prefix)
  std::vector<int> order(count);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return mem[x].nbb > mem[y].nbb; });

  const int slot = b->next;
  b->next = (b->next + 1) % kSlots;
  if (b->used[slot]) {
    cudaError_t e = cudaEventSynchronize(b->ev[slot]);
    if (e != cudaSuccess) return bcuda(e, "bt_batch_round: wait for member table slot");
  }
  unsigned char* h = b->h_slots + (size_t)slot * b->slot_bytes;
  unsigned char* d = b->d_slots + (size_t)slot * b->slot_bytes;
  Geo<T>* hg = reinterpret_cast<Geo<T>*>(h);
  MemberDesc<T>* hm = reinterpret_cast<MemberDesc<T>*>(h + b->geo_bytes);
  int* hoff = reinterpret_cast<int*>(h + b->geo_bytes + b->desc_bytes);
  const int stride = b->max_members + 1;
  int *o_tile = hoff, *o_fill = hoff + stride, *o_lfill = hoff + 2 * stride, *o_diag = hoff + 3 * stride;

  std::vector<const bt_plan*> plans;
  o_tile[0] = o_fill[0] = o_lfill[0] = o_diag[0] = 0;
  int any_diag = 0;
  for (int q = 0; q < count; ++q) {
    const bt_member& u = mem[order[q]];
    const bt_plan* p = u.plan;
    int gi = (int)(std::find(plans.begin(), plans.end(), p) - plans.begin());
    if (gi == (int)plans.size()) {
      if (gi == kMaxGeo) return bfail(BT_EINVAL, "bt_batch_round: more than 16 distinct plans in one call");
      plans.push_back(p);
      // the member plan's constant blocks for the batch's tile shape, built once per plan
      const int rc = ensure_const_blocks_any(u.plan, b->tile, s);
      if (rc != BT_OK) return rc;
      hg[gi] = p->geo_tile<T>(b->tile);
    }
    const ScratchLayout L = scratch_layout(p, rk);
    char* sc = (char*)u.scratch;
    MemberDesc<T>& md = hm[q];
    md.x0[0] = (const T*)u.in.h0;
    md.x0[1] = (const T*)u.in.ub;
    md.x0[2] = (const T*)u.in.vb;
    md.b0[0] = (const T*)u.in.h0p;
    md.b0[1] = (const T*)u.in.ubp;
    md.b0[2] = (const T*)u.in.vbp;
    md.x[0] = (T*)u.out.h0;
    md.x[1] = (T*)u.out.ub;
    md.x[2] = (T*)u.out.vb;
    for (int k = 0; k < 3; ++k) {
      md.y[k] = (T*)(sc + k * L.field);
      md.z[k] = rk == 3 ? (T*)(sc + (3 + k) * L.field) : nullptr;
    }
    md.fx = (T*)(sc + L.nfields * L.field);
    const bool dg = u.out.diag[0] != nullptr;
    for (int k = 0; k < 10; ++k) md.diag[k] = dg ? (T*)u.out.diag[k] : nullptr;
    md.dtb = u.dtb;
    md.geo = gi;
    md.nbb = u.nbb;
    const Tiling t = make_tiling(b->tile, p->n);
    o_tile[q + 1] = o_tile[q] + 6 * t.tiles_per_face();
    o_fill[q + 1] = o_fill[q] + 6 * p->nh;
    o_lfill[q + 1] = o_lfill[q] + (dg ? 6 * p->nh : 0);
    o_diag[q + 1] = o_diag[q] + (dg ? 6 * p->m * p->m : 0);
    any_diag |= dg ? 1 : 0;
  }
  cudaError_t e = cudaMemcpyAsync(d, h, b->slot_bytes, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return bcuda(e, "bt_batch_round: upload member table");

  BatchArgs<T> a;
  a.geos = reinterpret_cast<const Geo<T>*>(d);
  a.mem = reinterpret_cast<const MemberDesc<T>*>(d + b->geo_bytes);
  const int* doff = reinterpret_cast<const int*>(d + b->geo_bytes + b->desc_bytes);
  a.off.tile = doff;
  a.off.fill = doff + stride;
  a.off.lfill = doff + 2 * stride;
  a.off.diag = doff + 3 * stride;
  a.count = count;
  a.rk = rk;
  a.max_nbb = mem[order[0]].nbb;
  a.any_diag = any_diag;
  a.bar = b->d_flags;
  a.err = (int*)(b->d_flags + 1);
  a.spin_limit = b->spin_limit;
  const int nfill = o_fill[count] + o_lfill[count];
  const int ndiag = o_diag[count];

  if (b->mode == BT_MODE_PERSISTENT) {
    if ((e = cudaMemsetAsync(b->d_flags, 0, sizeof(unsigned), s)) != cudaSuccess)
      return bcuda(e, "bt_batch_round: reset barrier");
    e = launch_batch_round<T>(a, b->tile, o_tile[count], b->max_ctas, s, &b->last_grid);
    if (e == cudaErrorInvalidValue)
      return bfail(BT_EINVAL, "bt_batch_round: persistent mode takes at most 2^31 barrier arrivals per round "
                              "(2 x stages x substeps x CTAs): use fewer substeps per round or stream mode");
    if (e != cudaSuccess) return bcuda(e, "bt_batch_round: persistent launch");
  } else {
    const int nst = rk == 2 ? 2 : 3;
    int act = count;
    for (int step = 0; step < a.max_nbb; ++step) {
      while (act > 0 && hm[act - 1].nbb <= step) --act;
      for (int st = 0; st < nst; ++st)
        for (int uv = 0; uv < 2; ++uv) {
          e = launch_batch_phase<T>(a, b->tile, uv != 0, step, st, act, o_tile[act], s);
          if (e != cudaSuccess) return bcuda(e, "bt_batch_round: phase launch");
        }
    }
    if ((e = launch_batch_end<T>(a, nfill, ndiag, s)) != cudaSuccess) return bcuda(e, "bt_batch_round: halo fill");
  }
  if ((e = cudaEventRecord(b->ev[slot], s)) != cudaSuccess) return bcuda(e, "bt_batch_round: record slot event");
  b->used[slot] = true;
  return BT_OK;
}

}  // namespace

extern "C" {

int bt_member_scratch_bytes(bt_plan* plan, int rk, unsigned long long* bytes) {
  if (!plan || !bytes) return bfail(BT_EINVAL, "bt_member_scratch_bytes: NULL argument");
  if (rk != 2 && rk != 3) return bfail(BT_EINVAL, "bt_member_scratch_bytes: rk must be 2 or 3");
  *bytes = scratch_layout(plan, rk).total;
  return BT_OK;
}

int bt_batch_destroy(bt_batch* b) {
  if (!b) return BT_OK;
  int dev0 = 0;
  cudaGetDevice(&dev0);
  cudaSetDevice(b->device);
  for (int k = 0; k < kSlots; ++k)
    if (b->ev[k]) {
      cudaEventSynchronize(b->ev[k]);
      cudaEventDestroy(b->ev[k]);
    }
  cudaFree(b->d_slots);
  cudaFreeHost(b->h_slots);
  cudaFree(b->d_flags);
  cudaSetDevice(dev0);
  delete b;
  return BT_OK;
}

int bt_batch_create(int dtype, int max_members, bt_batch** out) {
  if (!out) return bfail(BT_EINVAL, "bt_batch_create: NULL argument");
  *out = nullptr;
  if (dtype != BT_F64 && dtype != BT_F32) return bfail(BT_EINVAL, "bt_batch_create: dtype must be BT_F64 or BT_F32");
  if (max_members < 1 || max_members > 65536)
    return bfail(BT_EINVAL, "bt_batch_create: max_members must be in [1, 65536]");
  bt_batch* b = new bt_batch;
  b->dtype = dtype;
  b->max_members = max_members;
  cudaGetDevice(&b->device);
  const size_t gsz = dtype == BT_F64 ? sizeof(Geo<double>) : sizeof(Geo<float>);
  const size_t msz = dtype == BT_F64 ? sizeof(MemberDesc<double>) : sizeof(MemberDesc<float>);
  b->geo_bytes = align256(kMaxGeo * gsz);
  b->desc_bytes = align256((size_t)max_members * msz);
  b->off_bytes = align256(4 * sizeof(int) * ((size_t)max_members + 1));
  b->slot_bytes = b->geo_bytes + b->desc_bytes + b->off_bytes;
  cudaError_t e = dtype == BT_F64 ? prime_batch<double>() : prime_batch<float>();
  if (e != cudaSuccess) {
    bt_batch_destroy(b);
    return bcuda(e, "bt_batch_create: kernel attributes");
  }
  if ((e = cudaMalloc(&b->d_slots, kSlots * b->slot_bytes)) != cudaSuccess ||
      (e = cudaHostAlloc(&b->h_slots, kSlots * b->slot_bytes, cudaHostAllocDefault)) != cudaSuccess ||
      (e = cudaMalloc(&b->d_flags, 2 * sizeof(unsigned))) != cudaSuccess ||
      (e = cudaMemset(b->d_flags, 0, 2 * sizeof(unsigned))) != cudaSuccess) {
    bt_batch_destroy(b);
    return bfail(BT_ENOMEM, std::string("bt_batch_create: allocation: ") + cudaGetErrorString(e));
  }
  std::memset(b->h_slots, 0, kSlots * b->slot_bytes);
  for (int k = 0; k < kSlots; ++k)
    if ((e = cudaEventCreateWithFlags(&b->ev[k], cudaEventDisableTiming)) != cudaSuccess) {
      bt_batch_destroy(b);
      return bcuda(e, "bt_batch_create: events");
    }
  *out = b;
  return BT_OK;
}

int bt_batch_set_mode(bt_batch* b, int mode) {
  if (!b) return bfail(BT_EINVAL, "bt_batch_set_mode: NULL batch");
  if (mode != BT_MODE_PERSISTENT && mode != BT_MODE_STREAM)
    return bfail(BT_EINVAL, "bt_batch_set_mode: mode must be BT_MODE_PERSISTENT or BT_MODE_STREAM");
  b->mode = mode;
  return BT_OK;
}

int bt_batch_set_tile(bt_batch* b, int ti, int tj) {
  if (!b) return bfail(BT_EINVAL, "bt_batch_set_tile: NULL batch");
  if (!tile_cfg_supported({ti, tj})) return bfail(BT_EINVAL, "bt_batch_set_tile: unsupported tile shape");
  b->tile = {ti, tj};
  return BT_OK;
}

int bt_batch_set_option(bt_batch* b, int key, long long value) {
  if (!b) return bfail(BT_EINVAL, "bt_batch_set_option: NULL batch");
  switch (key) {
    case BT_OPT_MAX_CTAS:
      if (value < 0 || value > (1 << 20)) return bfail(BT_EINVAL, "bt_batch_set_option: max_ctas out of range");
      b->max_ctas = (int)value;
      return BT_OK;
    case BT_OPT_SPIN_LIMIT:
      if (value < -1) return bfail(BT_EINVAL, "bt_batch_set_option: spin limit must be >= -1");
      b->spin_limit = value;
      return BT_OK;
    default:
      return bfail(BT_EINVAL, "bt_batch_set_option: unknown option");
  }
}

long long bt_batch_get_info(bt_batch* b, int key) {
  if (!b) return -1;
  if (key == BT_INFO_LAST_GRID) return b->last_grid;
  return -1;
}

int bt_batch_round(bt_batch* b, const bt_member* members, int count, int rk, void* stream) {
  if (!b || !members) return bfail(BT_EINVAL, "bt_batch_round: NULL argument");
  if (count < 1 || count > b->max_members)
    return bfail(BT_EINVAL, "bt_batch_round: count must be in [1, max_members] (" + std::to_string(b->max_members) + ")");
  if (rk != 2 && rk != 3) return bfail(BT_EINVAL, "bt_batch_round: rk must be 2 or 3");
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev != b->device) return bfail(BT_EINVAL, "bt_batch_round: the batch belongs to another device");
  long long tiles = 0;
  for (int q = 0; q < count; ++q) {
    const bt_member& u = members[q];
    const std::string who = "bt_batch_round: member " + std::to_string(q) + ": ";
    if (!u.plan) return bfail(BT_EINVAL, who + "NULL plan");
    if (u.plan->dtype != b->dtype) return bfail(BT_EINVAL, who + "plan dtype differs from the batch's");
    if (u.plan->device != b->device) return bfail(BT_EINVAL, who + "plan belongs to another device");
    if (u.nbb < 1) return bfail(BT_EINVAL, who + "nbb must be >= 1");
    const void* ptrs[10] = {u.in.h0, u.in.h0p, u.in.ub, u.in.vb, u.in.ubp, u.in.vbp,
                            u.out.h0, u.out.ub, u.out.vb, u.scratch};
    for (int k = 0; k < 10; ++k)
      if (!ptrs[k]) return bfail(BT_EINVAL, who + "NULL state or scratch pointer");
    if (((uintptr_t)u.scratch & 255) != 0) return bfail(BT_EINVAL, who + "scratch must be 256-byte aligned");
    if (u.out.h0 == u.in.h0 || u.out.ub == u.in.ub || u.out.vb == u.in.vb || u.out.h0 == u.in.h0p ||
        u.out.ub == u.in.ubp || u.out.vb == u.in.vbp)
      return bfail(BT_EINVAL, who + "outputs must not alias inputs");
    if (u.out.diag[0])
      for (int k = 1; k < 10; ++k)
        if (!u.out.diag[k]) return bfail(BT_EINVAL, who + "diag[0] set but diag[" + std::to_string(k) + "] is NULL");
    const Tiling t = make_tiling(b->tile, u.plan->n);
    tiles += 6LL * t.tiles_per_face();
  }
  if (tiles > (1LL << 30)) return bfail(BT_EINVAL, "bt_batch_round: too many tiles in one call");
  cudaStream_t s = (cudaStream_t)stream;
  return b->dtype == BT_F64 ? batch_round<double>(b, members, count, rk, s)
                            : batch_round<float>(b, members, count, rk, s);
}

int bt_batch_check_device_error(bt_batch* b) {
  if (!b) return bfail(BT_EINVAL, "bt_batch_check_device_error: NULL batch");
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return bcuda(e, "bt_batch_check_device_error: synchronize");
  unsigned flags[2];
  if ((e = cudaMemcpy(flags, b->d_flags, sizeof(flags), cudaMemcpyDeviceToHost)) != cudaSuccess)
    return bcuda(e, "bt_batch_check_device_error: read flag");
  if (flags[1] != 0) {
    cudaMemset(b->d_flags + 1, 0, sizeof(unsigned));
    if (flags[1] & kErrBarrierTimeout)
      return bfail(BT_EDEVICE, "batched round: grid barrier wait exceeded its poll limit; the round was abandoned");
    return bfail(BT_EDEVICE, "device error flag " + std::to_string(flags[1]));
  }
  return BT_OK;
}

}  // extern "C"
