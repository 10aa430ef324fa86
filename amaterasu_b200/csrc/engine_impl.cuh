// Internal layout of the engine object shared by the engine's translation units.
#pragma once
#include "common.cuh"

#include <cuda.h>

#include <vector>

namespace ama {

struct AxisPlan { int n, A, B; };

struct DeviceTables {
  int* plane_x = nullptr;      // [nslots]
  int* slot_of_x = nullptr;    // [n1] -> slot or -1
  int2* entries = nullptr;     // [sum npw]: (g, y*n3+z) grouped by (k, slot)
  int* entry_start = nullptr;  // [nk*(nslots+1)]
  int* rows = nullptr;         // concatenated y rows per (k, slot)
  int* row_start = nullptr;    // [nk*(nslots+1)]
  int64_t* pw_off = nullptr;   // [nk+1]
  int* npw = nullptr;          // [nk]
  double* kin64 = nullptr;     // [sum npw]
  float* kin32 = nullptr;
  void* tw[2][3][2] = {};      // [prec][axis][0 backward,1 forward]
  void* proj[2] = {};          // [prec] B, k-major (nproj, npw_k) blocks
  void* dproj[2] = {};         // [prec] D.B
  double* v64 = nullptr;       // [nspin][N] permuted, /N
  float* v32 = nullptr;
};

// Tensor-core (split-TF32) nonlocal path of the complex64 engine.
struct NlTcState {
  bool ready = false;
  int kp = 0;        // padded K of the projection (2*max npw, multiple of 32)
  int p2 = 0;        // padded rows of the real-expanded projectors (2*nproj, multiple of 128)
  int k2 = 0;        // padded K of the application (2*nproj, multiple of 32)
  int mp = 0;        // padded rows of the application (2*max npw, multiple of 128)
  float* bx[2] = {};   // hi/lo [nk][p2][kp]
  float* dxt[2] = {};  // hi/lo [nk][mp][k2]
  CUtensorMap map_bx[2], map_dxt[2];
  // per-call scratch (grown on demand); maps cached for (k_count, nbp)
  float* psi[2] = {};  size_t psi_bytes = 0;
  float* q[2] = {};    size_t q_bytes = 0;
  float* part = nullptr; size_t part_bytes = 0;
  int cached_kcount = -1, cached_nbp = -1;
  CUtensorMap map_psi[2], map_q[2];
  int* err = nullptr;
};

}  // namespace ama

using namespace ama;

struct AmaEngine {
  AxisPlan ax[3];
  int64_t N = 0;
  int nk = 0, nspin = 1, nproj = 0, nslots = 0;
  // the used x-planes are exactly x <= slot_hp and x >= n1 - slot_hn (else both -1)
  int slot_hp = -1, slot_hn = -1;
  uint32_t precisions = 0;
  std::vector<int> npw;
  std::vector<int64_t> pw_off;
  int max_npw = 0;
  int max_rows = 0;
  DeviceTables d;
  bool has_potential = false;
  // workspaces (grown on demand)
  void* work[2] = {};
  size_t work_bytes[2] = {};
  void* ws_proj[2] = {};       // P = psi B^H
  size_t ws_proj_bytes[2] = {};
  void* ws_part[2] = {};       // split-K partials
  size_t ws_part_bytes[2] = {};
  double* ws_dens = nullptr;   // permuted density accumulator
  size_t ws_dens_bytes = 0;
  const void* stage_fn[2][4] = {};  // [prec][stage A, B, C, density B] (grid-specialised)
  int zsplit[2] = {1, 1};           // [prec] z halves per stage-B slab
  bool regb[2] = {false, false};    // [prec] stage B with register-resident x columns
  const void* b_variant[2][5] = {};  // [prec] stage B variants compiled for the grid
  int b_zsplit[2][5] = {};           // [prec] z split of each variant's shared-memory slab
  int bthreads[2] = {1, 1};          // [prec] threads per (y, z) column of the register stage B
  const void* ac_variant[2][2][2] = {};  // [prec][variant][stage A, C] compiled for the grid
  int ac_threads_of[2][2] = {};          // [prec][variant] threads per CTA of those stages
  int ac_threads[2] = {256, 256};        // [prec] threads per CTA of the selected stages A and C
  NlTcState tc;
  bool use_tc = true;
  bool dav_graphs = true;  // ama_davidson replays recurring iteration segments as CUDA graphs
  // FP64 grid transforms (Hartree, Kerker): reciprocal-space filters in the engine's
  // permuted order, and the complex work grid of ama_grid_filter / ama_grid_fft_forward.
  // Both live on the engine's device; calls on one engine from different streams race on
  // the work grid.
  double* grid_filt[4] = {};
  double2* grid_work = nullptr;
  size_t grid_work_bytes = 0;
  int device = 0;
};

namespace ama {
int nl_tc_setup(AmaEngine* e);
// phase 0: split psi, project, reduce (P -> split Q); phase 1: apply (hpsi += Q D B);
// phase 2: both in order
int nl_tc_run(AmaEngine* e, int k_first, int k_count, int nbands, const float2* psi, float2* hpsi,
              cudaStream_t s, int phase = 2);
int nl_tc_apply(AmaEngine* e, int k_first, int k_count, int nbands, float2* hpsi, cudaStream_t s, int ntile,
                int bn);
void nl_tc_free(AmaEngine* e);
// look up the allocation-free grid array on the current device (once per device)
int noalloc_prepare();
}  // namespace ama


