// Internal (host) definitions of libcetagpu: the handle and its device state.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>
#include "../../include/cetasim_gpu.h"
#include "track_math.cuh"

namespace cg {

constexpr int kTile = 256;            // particles per tile == threads per CTA

constexpr int kMomChunkTiles = 4;     // tiles per CTA of the moments kernel
constexpr int kMaxPipeGroups = 16;    // segments of the pipelined ion pass

struct BunchDev {
  int n, tile_off, n_tiles, harm, gap;
  int chunk_off, n_chunks;  // moments chunks of kMomChunkTiles tiles
  double ne, q_macro;
};

// Broadband impedance (cg_config::bbi), set up at cg_create.
constexpr int kBbiHalf = 25;  // half width of the K = 51 Gaussian filter (MPBunch.cpp:2376)
struct BbiParams {
  int td = 0;                  // 1: time domain (wake table), 0: frequency domain
  int sim[5] = {0, 0, 0, 0, 0};  // planes Z, Dx, Dy, Qx, Qy
  int nbins = 0;               // profile bins: 2 n - 1 (frequency), int(rfLen / dz) (time)
  int nw = 0;                  // wake samples per plane
  int s0 = 0, s1 = 0;          // the filter runs over the bins [s0, s1)
  int wcap = 0;                // bins kept per bunch: min(CG_BBI_MAX_BINS, nbins) + 2 kBbiHalf
  double zmin = 0, dz = 0;     // left edge of bin 0 (frequency domain: its centre), width
  double energy = 0, beta2 = 0;  // electronBeamEnergy, pow(rBeta, 2)
  double beta_x = 0, beta_y = 0; // twissBetaX[0], twissBetaY[0]
  double g[2 * kBbiHalf + 1];  // normalised Gaussian filter kernel
};

// Space charge (cg_config::flag_sc), set up at cg_create.
struct ScParams {
  int flag = 0;                // 1 Bassetti-Erskine slices, 2 2.5-D PIC, 3 linear
  int nx = 0, ny = 0, nz = 0;  // mesh nodes (PIC) and slices
  int acc_per_slice = 0;       // accumulators per slice: nx ny (PIC) or 4
  double range = 10.0;         // mesh half-width in rms sizes (PIC3D.h:62, PIC3D.cpp:152)
  double p0 = 0;               // beta0 gamma0 of the reference particle (PIC2D.cpp)
};

// Ion cloud of one (IP, species): ping-pong buffers of capacity `cap`.
struct CloudDev {
  double* x[2];
  double* y[2];
  double* vx[2];
  double* vy[2];
  double* fx;  // velocity kick of the last bunch on each ion (ionAccumuFx, MPBunch.cpp:1149)
  double* fy;
  int cap;
};

// Device-side per-(IP, species) ion state that persists across launches.
struct CloudState {
  int n;         // ionAccumuNumber
  int cur;       // which ping-pong buffer holds the cloud
  double aver_x, aver_y, rms_x, rms_y;  // IonRMSCal (stale when n <= 1)
  double macro_charge;
};

// Parameters of the ion chain kernel that do not change between launches.
struct ChainParams {
  double cross_section[CG_MAX_SPECIES], gas_percent[CG_MAX_SPECIES], mass_number[CG_MAX_SPECIES];
  double loss_boundary;
  double circ_ring, harmonics;  // ion drift over a gap: v C/h gap/c (LIP.cpp:1172-1173)
  double r_gamma;
  int n_species, macro_per_ip, max_ions, n_bunches;
  uint64_t seed;
};

// Section data the ion chain of one IP needs.
struct ChainSection {
  double pressure, temperature, length, aperture_x, aperture_y;
};

// Scratch of the ion chain (one IP at a time, reused across IPs): per-bunch
// constants and births from k_ion_prep, per-step partial sums and trajectory
// end states from k_ion_walk.
struct IonWalk {
  double* births = nullptr;   // P x M x NM x (x, y)
  FieldPrep* prep = nullptr;  // M: field constants of each bunch
  double* bunch = nullptr;    // M x (mean x, mean y, drift time to the next bunch)
  double* spec = nullptr;     // P x M x (macro-ion charge, ion-side coefficient)
  double* bound = nullptr;    // loss bounds (x, y)
  double* part = nullptr;     // P x M x grid x (count, sum x, sum y, sum x^2, sum y^2)
  double* traj = nullptr;     // P x 6 x tcap: x, y, vx, vy after the walk, last kick fx, fy
  uint8_t* alive = nullptr;   // P x tcap
  double* carry = nullptr;    // P x (centroid x, y carried between steps, last rms x, y)
  int64_t tcap = 0;           // trajectories per species: cloud capacity + M x NM
  int grid = 0;               // CTAs of k_ion_walk per species
};

struct DeviceBufs {
  double* c = nullptr;          // 6 x npad SoA
  uint8_t* surv = nullptr;      // npad
  int* tile_bunch = nullptr;    // n_tiles
  int* chunk_bunch = nullptr;   // n_chunks: bunch of each moments chunk
  int4* chunk_loc = nullptr;    // n_chunks: (bunch, first tile, chunk of the bunch, valid slots)
  BunchDev* bunch = nullptr;    // M
  MomPartial* wpartials = nullptr; // n_chunks x 8: per-warp moment partials
  unsigned* counters = nullptr;    // M (+ spare)
  BunchMomDev* mom = nullptr;      // M
  int* loss_count = nullptr;       // M
  int* status = nullptr;           // device status word(s)
  int* turn = nullptr;             // device turn counter (graph replays)
  // ion clouds
  CloudDev* clouds = nullptr;      // K x P (device array of buffer pointers)
  CloudState* cloud_state = nullptr;  // K x P
  CloudRec* rec = nullptr;         // K x M x P
  FieldPrep* rec_prep = nullptr;   // K x M x P: field constants of each record's Gaussian
  double* ion_totals = nullptr;    // K (charge), used by cg_ion_totals
  IonWalk iw;
  // bunch-sharded runs: moments of the local bunches out, of all bunches in
  BunchMomDev* mom_send = nullptr;  // max local bunches
  BunchMomDev* mom_all = nullptr;   // ranks x max local bunches
  int* sh_off = nullptr;            // ranks: first bunch of each rank
  int* sh_cnt = nullptr;            // ranks: bunches of each rank
  // field surrogate
  float* sur_w = nullptr;                 // FP32 parameters (null: exact kicks)
  unsigned long long* sur_audit = nullptr;  // audit maxima (double bit patterns)
  // long-range wake
  double* lr_tab = nullptr;        // 3 x np
  double* lr_hist = nullptr;       // turns x 3 x M ring buffer
  int* lr_head = nullptr;
  double* lr_force = nullptr;      // M x 3
  // FIR
  double* fir_hist = nullptr;      // order x 3 x M ring buffer
  int* fir_head = nullptr;
  double* fir_kick = nullptr;      // M x 3
  double* fir_coeff = nullptr;     // 3 x order
  // short-range wake
  double* sr_geom = nullptr;       // M x 2 (zlo, dz)
  int* sr_counts = nullptr;        // M x B
  double* sr_sumx = nullptr;       // M x B
  double* sr_sumy = nullptr;       // M x B
  double* sr_lag = nullptr;        // M x (2B-1)
  double* sr_pot = nullptr;        // M x B (z plane, persistent)
  double* sr_green = nullptr;      // resonators x 1000 (u-independent factors)
  double* sr_green_t = nullptr;    // the same for the transverse planes x, y
  double* sr_potxy = nullptr;      // M x 2 x B transverse potentials (persistent, cg_set_sr_potentials)
  // coupled-bunch mode history (cg_cbm_*): records x kCbmRecord x M
  double* cbm = nullptr;
  // cavities with beam loading (rfMode 1)
  double* res_state = nullptr;     // CG_MAX_CAVITIES x 6: vbAccum, resGenVol, resGenIg
  double* rf_zr = nullptr;         // M x 2: z range of the RF step
  int* rf_counts = nullptr;        // M x bins
  double* rf_kick = nullptr;       // loading cavities x M x bins x 2
  double* rf_fbk = nullptr;        // loading cavities x M: direct-feedback kicks
  double* rf_work = nullptr;       // work buffers of the cavities' recurrence
  double* rf_info = nullptr;       // M x CG_MAX_CAVITIES x 8: BunchRFModeInfo
  // broadband impedance
  double* bbi_w = nullptr;         // 5 x nw wake samples (planes Z, Dx, Dy, Qx, Qy)
  int* bbi_lo = nullptr;           // M: lowest bin holding a particle (INT_MAX between calls)
  int* bbi_hi = nullptr;           // M: highest (-1 between calls)
  unsigned long long* bbi_amax = nullptr;  // M x 2: largest |x|, |y| (bit patterns)
  int* bbi_cnt = nullptr;          // M x wcap per-bin counts (zero between calls)
  unsigned long long* bbi_sxy = nullptr;  // M x 2 x wcap fixed-point sums of x, y
  double* bbi_pot = nullptr;       // M x 6 x wcap: profile and potentials of the last kick
  int2* bbi_win = nullptr;         // M: first bin and bin count of bbi_pot
  // space charge
  double* sc_geom = nullptr;       // M x 11: slices, mesh, fixed-point scales
  int* sc_cnt = nullptr;           // M x nz particles per slice
  unsigned long long* sc_acc = nullptr;  // M x nz x acc_per_slice fixed-point sums
  double* sc_field = nullptr;      // M x nz x 2 x nx x ny mesh field (PIC)
  int* sc_slice_of = nullptr;      // npad: each particle's slice (PIC)
  int* sc_list = nullptr;          // npad: particle indices grouped by bunch and slice (PIC)
  int* sc_start = nullptr;         // M x nz: first list entry of each slice (PIC)
  int* sc_cursor = nullptr;        // M x nz: fill cursors (PIC)
  double* sc_sin = nullptr;        // nx x nx + ny x ny: 2 sin(pi (i + 1)(k + 1) / (n + 1))
  // phase advance of the tracked bunches: slot per bunch (-1 untracked),
  // per slot 6 x n (previous angles x, y, z; accumulated x, y, z)
  int* phase_slot = nullptr;
  double** phase_ptr = nullptr;
  // scratch
  double* scratch = nullptr;
  size_t scratch_bytes = 0;
};

constexpr int kCbmRecord = 15;  // doubles per bunch in one coupled-bunch mode record

// Coupled-bunch mode record constants (cbm.cu): per plane x, y, z
struct CbmParams {
  double sqrt_beta[3], alpha_sqrt[3];  // sqrt(beta), alpha / sqrt(beta) at section 0 (z: alpha 0)
  double tune[3];
  int H, M;
};

struct TraceMark {
  int kind, stream, ip, seg;
};

struct Handle {
  cg_config cfg;
  std::vector<cg_section> sections;
  std::vector<SectionDev> sec_dev_host;
  SectionDev* sec_dev = nullptr;  // device copy (K)
  RingDev ring;
  ChainParams chain;
  int device = 0;
  cudaStream_t stream = nullptr;
  int K = 0, M = 0, P = 1;
  int n_tiles = 0;
  int n_chunks = 0;
  int64_t npad = 0;
  std::vector<int> n_macro, harm, gap, tile_off, chunk_off;
  // pipelined turn: the ion walk of an IP in `pipe_groups` segments of bunches;
  // records, kicks and maps of a segment run on `side` while the next segment
  // walks
  int cbm_cap = 0, cbm_n = 0;  // coupled-bunch mode history: capacity, records made
  double sr_rw_coeff = 0.0;    // short-range resistive-wall coefficient (0: no sectors)
  BbiParams bbi;               // broadband impedance (cfg.bbi.flag)
  ScParams sc;                 // space charge (cfg.flag_sc)
  bool sr_xy = false;          // SR wake: the transverse potentials too (the reference's file)
  std::vector<int> phase_bunches;  // bunches whose particles' phase advance is tracked
  std::vector<double*> phase_bufs; // their device buffers (6 x n each)
  std::vector<double> bbi_table;  // the copy of cfg.bbi.table
  int pipe_groups = 4;
  // trajectories per walk CTA (8, 16, 32, 64): smaller CTAs spread the
  // walk's FP64 work over more SMs and find room sooner while the kicks and
  // maps of earlier segments fill the GPU
  int walk_ions = 64;
  bool pipe_ramp = false;  // last walk segment half as long as the others
  bool walk_reserve = false;  // walk CTAs take their SM's whole shared memory
  // turn trace (cg_trace_turn): marks and their timing events
  std::vector<TraceMark>* trace = nullptr;
  std::vector<cudaEvent_t> trace_ev;
  cudaStream_t side = nullptr;   // records and kicks of the segments
  cudaStream_t side2 = nullptr;  // maps of the segments (kick g + 1 overlaps map g)
  std::vector<cudaEvent_t> pipe_ev;  // kMaxPipeGroups + 1: walked segments, then the join
  std::vector<cudaEvent_t> kick_ev;  // kMaxPipeGroups + 1: kicked segments, then the join
  std::vector<double> ne;
  DeviceBufs d;
  int lr_np = 0;
  double lr_dt = 0;
  int fir_order = 0;
  double fir_limit = 0;
  bool beam_set = false;
  int ion_cap = 0;
  cudaGraphExec_t turn_graph = nullptr;
  int kick_variant = 0;         // autotuned shape of the kick kernel
  bool fuse_kick = false;       // autotuned: kick inside the map pass
  bool map_async = false;       // autotuned: the map pass with the next chunk in flight
  int sh_rank = 0, sh_world = 1;  // bunch sharding over ranks (cg_set_shard)
  int sh_j0 = 0, sh_j1 = 0, sh_maxlocal = 0;
  void* nccl_comm = nullptr;
  int sur_audit_every = 0;     // turns between exact audits of the surrogate (0: none)
  int sur_audits = 0;
  double sur_audit_last = 0, sur_audit_worst = 0;
  std::string err;
};

}  // namespace cg

struct cg_handle {
  cg::Handle h;
};
