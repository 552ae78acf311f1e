// Bunch-sharded runs over several GPUs, one process per GPU.
//
// Bunches are independent except through small per-bunch aggregates, so each
// rank holds a contiguous range of bunches (balanced by macroparticle count)
// and tracks only those particles.  What couples the ranks is the per-bunch
// moments: the ion chain at an IP reads the centroid and size of every bunch
// (and the largest size, for the ion loss bound), and the long-range wake and
// the FIR feedback read every bunch's centroid.  After each moments pass the
// ranks therefore all-gather the moments (an NCCL all-gather on the handle's
// stream, captured in the turn graph like the kernels); every rank then runs
// the same ion chain on the same inputs (deterministic: identical records on
// every rank) and kicks its own bunches.
//
// NCCL is loaded at run time (the library has no link-time dependency on it);
// a process that already loaded it (PyTorch with its NCCL backend) shares
// that copy.  Otherwise the system's libnccl.so.2 is opened, and a library
// loaded later that needs a newer NCCL under the same soname (PyTorch) would
// find the older one: such a process loads PyTorch first.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nccl.h>
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>
#include "kernels.cuh"

namespace cg {

namespace {

struct NcclApi {
  bool tried = false, ok = false;
  ncclResult_t (*get_unique_id)(ncclUniqueId*) = nullptr;
  ncclResult_t (*comm_init_rank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*all_gather)(const void*, void*, size_t, ncclDataType_t, ncclComm_t,
                             cudaStream_t) = nullptr;
  ncclResult_t (*comm_destroy)(ncclComm_t) = nullptr;
  const char* (*error_string)(ncclResult_t) = nullptr;
};

NcclApi& nccl() {
  static NcclApi api;
  if (api.tried) return api;
  api.tried = true;
  void* lib = dlopen("libnccl.so.2", RTLD_NOW | RTLD_NOLOAD);
  if (!lib) lib = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
  if (!lib) lib = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
  if (!lib) return api;
  api.get_unique_id = (decltype(api.get_unique_id))dlsym(lib, "ncclGetUniqueId");
  api.comm_init_rank = (decltype(api.comm_init_rank))dlsym(lib, "ncclCommInitRank");
  api.all_gather = (decltype(api.all_gather))dlsym(lib, "ncclAllGather");
  api.comm_destroy = (decltype(api.comm_destroy))dlsym(lib, "ncclCommDestroy");
  api.error_string = (decltype(api.error_string))dlsym(lib, "ncclGetErrorString");
  api.ok = api.get_unique_id && api.comm_init_rank && api.all_gather && api.comm_destroy &&
           api.error_string;
  return api;
}

}  // namespace

// Contiguous bunch ranges [j0[r], j1[r]) for `world` ranks with about equal
// macroparticle counts: rank r ends at the first bunch boundary where the
// running count reaches (r + 1) / world of the total (every rank gets at least
// one bunch when M >= world).
void shard_plan(const int* n_macro, int M, int world, int* j0, int* j1) {
  double total = 0;
  for (int j = 0; j < M; ++j) total += n_macro[j];
  int j = 0;
  double run = 0;
  for (int r = 0; r < world; ++r) {
    j0[r] = j;
    const double target = total * (r + 1) / world;
    const int must_leave = world - 1 - r;  // bunches the later ranks need at least
    while (j < M - must_leave && (r == world - 1 || run + 0.5 * n_macro[j] < target || j == j0[r])) {
      run += n_macro[j];
      ++j;
    }
    j1[r] = j;
  }
}

// The exchange layout of a plan: rank r owns bunches [j0[r], j1[r]) and
// sends its records as one slot of max_local records (padded), so the
// all-gather output holds rank r's records at slot r; j0 / cnt place them.
ShardLayout shard_layout(const int* n_macro, int M, int world) {
  ShardLayout L;
  L.j0.assign(world, 0);
  L.j1.assign(world, M);
  if (world > 1) shard_plan(n_macro, M, world, L.j0.data(), L.j1.data());
  L.cnt.resize(world);
  L.max_local = 0;
  for (int r = 0; r < world; ++r) {
    L.cnt[r] = L.j1[r] - L.j0[r];
    L.max_local = std::max(L.max_local, L.cnt[r]);
  }
  return L;
}

// Host form of the exchange's two local steps (the device runs the same
// layout with a copy and k_scatter_moments around the NCCL all-gather):
// pack copies this rank's records into its send slot (zero padding), unpack
// places every rank's slot of the gathered buffer at its bunches.
void shard_pack_host(const ShardLayout& L, int rank, const unsigned char* records, size_t rec,
                     unsigned char* send) {
  std::memset(send, 0, (size_t)L.max_local * rec);
  std::memcpy(send, records + (size_t)L.j0[rank] * rec, (size_t)L.cnt[rank] * rec);
}

void shard_unpack_host(const ShardLayout& L, const unsigned char* gathered, size_t rec,
                       unsigned char* records) {
  for (size_t r = 0; r < L.cnt.size(); ++r)
    std::memcpy(records + (size_t)L.j0[r] * rec, gathered + r * (size_t)L.max_local * rec,
                (size_t)L.cnt[r] * rec);
}

__global__ void k_scatter_moments(const BunchMomDev* __restrict__ all, BunchMomDev* mom,
                                  const int* __restrict__ off, const int* __restrict__ cnt,
                                  int world, int maxlocal) {
  const int r = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt[r]; i += gridDim.x * blockDim.x)
    mom[off[r] + i] = all[(size_t)r * maxlocal + i];
}

// All ranks: moments of every bunch from the owners' slices.
cudaError_t exchange_moments(Handle& h) {
  if (!h.nccl_comm) return cudaSuccess;
  const size_t nloc = (size_t)(h.sh_j1 - h.sh_j0);
  cudaError_t e = cudaMemcpyAsync(h.d.mom_send, h.d.mom + h.sh_j0, nloc * sizeof(BunchMomDev),
                                  cudaMemcpyDeviceToDevice, h.stream);
  if (e != cudaSuccess) return e;
  ncclResult_t r = nccl().all_gather(h.d.mom_send, h.d.mom_all,
                                     (size_t)h.sh_maxlocal * sizeof(BunchMomDev), ncclUint8,
                                     (ncclComm_t)h.nccl_comm, h.stream);
  if (r != ncclSuccess) return cudaErrorUnknown;
  dim3 grid((h.sh_maxlocal + 127) / 128, h.sh_world);
  k_scatter_moments<<<grid, 128, 0, h.stream>>>(h.d.mom_all, h.d.mom, h.d.sh_off, h.d.sh_cnt,
                                                 h.sh_world, h.sh_maxlocal);
  return cudaGetLastError();
}

std::string nccl_error(int r) {
  NcclApi& a = nccl();
  return a.ok ? a.error_string((ncclResult_t)r) : "NCCL not loaded";
}

int nccl_unique_id(void* out) {
  NcclApi& a = nccl();
  if (!a.ok) return -1;
  ncclUniqueId id;
  ncclResult_t r = a.get_unique_id(&id);
  if (r != ncclSuccess) return (int)r;
  std::memcpy(out, &id, sizeof id);
  return 0;
}

int nccl_comm_init(void** comm, int world, const void* id, int rank) {
  NcclApi& a = nccl();
  if (!a.ok) return -1;
  ncclUniqueId uid;
  std::memcpy(&uid, id, sizeof uid);
  ncclComm_t c = nullptr;
  ncclResult_t r = a.comm_init_rank(&c, world, uid, rank);
  if (r != ncclSuccess) return (int)r;
  *comm = c;
  return 0;
}

void nccl_comm_destroy(void* comm) {
  if (comm && nccl().ok) nccl().comm_destroy((ncclComm_t)comm);
}

bool nccl_available() { return nccl().ok; }

}  // namespace cg
