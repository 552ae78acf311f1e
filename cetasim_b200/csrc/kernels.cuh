// Kernel launchers of libcetagpu (host-callable, implemented in kernels.cu).
#pragma once
#include "cg_internal.h"

namespace cg {

// status word bits (DeviceBufs::status[0])
enum : int {
  kStatusIonOverflow = 1,
  kStatusTransmission = 2,
  kStatusLrRange = 4,
  kStatusIonBirth = 8,
  kStatusSurrogateWait = 16,  // a tensor-core completion wait gave up
  kStatusGaussCut = 64,       // an initial-distribution draw found no accepted sample
  kStatusBbiRange = 128,      // a particle outside the broadband-impedance profile
  kStatusBbiWide = 256,       // a bunch over more than CG_BBI_MAX_BINS profile bins
  kStatusScMesh = 512,        // a space-charge mesh from a zero rms size
};

// per-particle phase advance of the tracked bunches (cg_set_phase_track)
cudaError_t launch_phase_init(Handle& h);
// before the last section's map, for the tracked bunches among [ja, jb)
cudaError_t launch_phase_adv(Handle& h, int ja, int jb, cudaStream_t s = nullptr);

// space charge (sc.cu)
cudaError_t launch_space_charge(Handle& h, int k);
size_t sc_solve_smem(const ScParams& p);
cudaError_t prepare_sc(const ScParams& p);

// broadband impedance (bbi.cu)
cudaError_t launch_bbi(Handle& h);
size_t bbi_conv_smem(const BbiParams& p);
cudaError_t prepare_bbi(const BbiParams& p);
// w (5 x (2n - 1)) from the impedances X (5 x n, device) on stream st
cudaError_t bbi_wake_fd(const double2* d_X, int n, double* d_w, cudaStream_t st);

cudaError_t launch_moments(Handle& h, int k);
cudaError_t launch_map(Handle& h, int k);
cudaError_t launch_ion_chain(Handle& h, int k);
// the chain in pieces (the pipelined turn): prep, walk / records of the bunch
// steps [ja, jb), compaction
cudaError_t launch_ion_prep(Handle& h, int k);
cudaError_t launch_ion_walk(Handle& h, int k, int ja, int jb, cudaStream_t s);
cudaError_t launch_ion_records(Handle& h, int k, int ja, int jb, cudaStream_t s);
cudaError_t launch_ion_compact(Handle& h, int k, cudaStream_t s);
// walk CTAs for `tcap` trajectory slots at `ions` trajectories per CTA
int ion_walk_grid(int64_t tcap, int ions);
// per device, once: the shared-memory reservation of each walk shape
cudaError_t prepare_ion_walk();
cudaError_t launch_ion_kick(Handle& h, int k);
// the kick of the tiles [tile_a, tile_b) (tile_b < 0: all) on stream s (null: h.stream)
cudaError_t launch_ion_kick_variant(Handle& h, int k, int v, int tile_a = 0, int tile_b = -1,
                                    cudaStream_t s = nullptr);
int kick_variants();
void kick_variant_shape(int v, int* threads, int* min_ctas);
// (ion kick of IP k if `kick`) + map of section k + moments at section
// `mom_section` (if >= 0), over the moments chunks [chunk_a, chunk_b)
// (chunk_b < 0: all) on stream s (null: h.stream)
cudaError_t launch_map_pass(Handle& h, int k, int mom_section, bool kick = false, int chunk_a = 0,
                            int chunk_b = -1, cudaStream_t s = nullptr);
// The same pass with the next chunk in flight: a persistent grid (two CTAs
// per SM) in which every thread stages its slots of the CTA's next chunk in
// shared memory by cp.async while it maps and reduces the current one.
cudaError_t launch_map_async(Handle& h, int k, int mom_section, bool kick = false,
                             int chunk_a = 0, int chunk_b = -1, cudaStream_t s = nullptr);
// the map pass of the turn: the asynchronous form when h.map_async is set
cudaError_t launch_map_turn(Handle& h, int k, int mom_section, bool kick = false,
                            int chunk_a = 0, int chunk_b = -1, cudaStream_t s = nullptr);
// per device, once: the dynamic shared memory of the asynchronous map pass
cudaError_t prepare_map_async();
enum LongFlags : unsigned {
  kLongRF = 1,
  kLongDrift = 2,
  kLongLoss = 4,
  kLongSynrad = 8,
  kLongLR = 16,
};
cudaError_t launch_long(Handle& h, unsigned flags);
// cavities with beam loading: z ranges and bins of the RF step, then the
// cavities' recurrence over the train (beam_loading.cu); k_long applies the
// kicks
cudaError_t launch_rf_beam_loading(Handle& h);
size_t rf_work_doubles(int n_bl, int M, int nb);
void resonator_init(const cg_config& cfg, const std::vector<int>& harm,
                    const std::vector<double>& ne, double* state, double* info);
cudaError_t launch_lr_compute(Handle& h);
cudaError_t launch_lr_kick(Handle& h);
cudaError_t launch_fir_compute(Handle& h);
cudaError_t launch_mark_lost(Handle& h, bool fir_kick, bool mark);
cudaError_t launch_sr_wake(Handle& h);
cudaError_t launch_turn_advance(Handle& h);
cudaError_t launch_gaussian(Handle& h, double emit_x, double emit_y, double sigma_z,
                            double sigma_dp, uint64_t seed);
cudaError_t launch_faddeeva(const double* zr, const double* zi, double* wr, double* wi, int64_t n,
                            bool general, cudaStream_t s);
cudaError_t launch_field(const double* x, const double* y, const double* sx, const double* sy,
                         double* fx, double* fy, int64_t n, cudaStream_t s);
// bunch sharding (shard.cu)
void shard_plan(const int* n_macro, int M, int world, int* j0, int* j1);
struct ShardLayout {
  std::vector<int> j0, j1, cnt;  // bunch range and count of each rank
  int max_local = 0;             // records per rank slot of the all-gather
};
ShardLayout shard_layout(const int* n_macro, int M, int world);
void shard_pack_host(const ShardLayout& L, int rank, const unsigned char* records, size_t rec,
                     unsigned char* send);
void shard_unpack_host(const ShardLayout& L, const unsigned char* gathered, size_t rec,
                       unsigned char* records);
cudaError_t exchange_moments(Handle& h);
int nccl_unique_id(void* out);
int nccl_comm_init(void** comm, int world, const void* id, int rank);
void nccl_comm_destroy(void* comm);
std::string nccl_error(int r);
bool nccl_available();

// coupled-bunch mode history and growth-rate fit (cbm.cu)
cudaError_t launch_cbm_record(Handle& h, const CbmParams& p, int rec);
cudaError_t launch_cbm_fit(Handle& h, int method, int M, int first, int dim, double interval,
                           double t0, double* rate);
// the Hilbert method over records [0, N): spec N x 3 x M scratch, ana the
// analytic signals, hamp the modes' amplitudes, babs |a| per bunch (N x 3 x M)
cudaError_t launch_cbm_hilbert(Handle& h, const CbmParams& p, int N, double2* spec, double2* ana,
                               double* hamp, double* harg, double* babs);
cudaError_t launch_cbm_fit_plain(Handle& h, const double* a, int M, int first, int dim,
                                 double interval, double t0, double* rate);

// field surrogate (surrogate.cu)
cudaError_t prepare_surrogate();
cudaError_t launch_sur_data(uint64_t seed, int64_t n, float* xin, float* tout, cudaStream_t s);
cudaError_t launch_sur_eval(const float* w, const float* xin, int64_t n, float* out, int* status,
                            cudaStream_t s);
cudaError_t launch_sur_step(const float* w, const float* xin, const float* tin, int64_t n,
                            int64_t row0, int batch, uint64_t mul, uint64_t add, float* part,
                            float* m, float* v, float* wmut, float lr, float bc1, float bc2,
                            double* loss, float* grad_out, int* status, cudaStream_t s,
                            float l4w = 0.0f, float* e2_sum = nullptr);
cudaError_t launch_ion_kick_sur(Handle& h, int k, int tile_a = 0, int tile_b = -1,
                                cudaStream_t s = nullptr);
cudaError_t launch_sur_audit(Handle& h, int k, unsigned long long* out);
cudaError_t upload_weideman_table_sur();

cudaError_t upload_weideman_table();      // every translation unit that evaluates w(z)
cudaError_t upload_weideman_table_ion();
// the copy of the w(z) table in sc.cu (the Bassetti-Erskine slice model)
cudaError_t upload_weideman_table_sc();

// Moments of one bunch held in the caller's device buffers, with the partials
// in a fixed file-scope device array (no allocation).  At most
// kNoAllocMaxTiles tiles of kTile particles per call.
constexpr int kNoAllocMaxTiles = 4096;
cudaError_t noalloc_scratch_address(double** ptr);
cudaError_t launch_moments_noalloc(const double* c, int64_t stride, const uint8_t* surv, int n,
                                   double beta_x, double beta_y, double* scratch,
                                   cg_bunch_moments* out, cudaStream_t s);
cudaError_t measure_fp64_peak(double* flops);
cudaError_t measure_field_chain_latency(double* us_per_step);
cudaError_t launch_eigen_sums(Handle& h, int j, double* out);

}  // namespace cg
