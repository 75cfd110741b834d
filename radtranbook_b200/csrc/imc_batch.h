// imc_batch.h — kernel arguments of the batched 1-D slab engine (imc_batch_* in
// include/imcb200.h).  One struct, passed by value to every batch kernel.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/imcb200.h"

struct BatchBank {
  float* p1; float* d1; float* w; float* t; int* cell;
};

struct BatchArgs {
  int K, n_cells;
  long long n_slots, max_tiles;
  double dt, theta;
  // problem
  const int* cell_off; const double* edges; const long long* slot_off; const uint64_t* seed;
  const long long* n_target; const long long* n_boundary; const long long* n_max;
  const double* face_T; const int* reflect; const double* op_a; const double* op_p; const double* cv;
  // state
  BatchBank bank[2];
  int* sel; uint32_t* step; long long* n_census;
  double* T; double* e; double* tr; double* dep; double* si; double* emitted; double* ledger;
  unsigned long long* stats; int* flags;
  // workspace: per cell
  int* cell_inst;        // [n_cells] instance of a cell
  float* ef;             // [n_cells + K] FP32 edges
  double* vol;           // [n_cells] dx
  float2* sass;          // [n_cells] (sigma_a, sigma_s) FP32
  double2* cellf;        // [n_cells] (1/V, 1/(sigma_a V dt) or -1/(V dt))
  double* emit_E;        // [n_cells]
  long long* emit_n;     // [n_cells]
  long long* emit_off;   // [n_cells + K] instance k: nc_k + 1 offsets from cell_off[k] + k
  float* emit_w;         // [n_cells]
  double* tilt;          // [n_cells] slab linear-T slope
  double* ecen; double* ew; double* ncopy;  // [n_cells] comb
  // workspace: per instance
  long long* n_side;     // [2K]
  float* w_side;         // [2K]
  long long* n_bank;     // [K] entries tracked this step
  long long* n_new;      // [K] new particles this step
  long long* census_cap; // [K] largest census the slot range holds next to a step's sources
  long long* live_pref;  // [K+1]
  long long* new_pref;   // [K+1]
  long long* inst_pref;  // [K+1] exclusive prefix of comb copies per instance
  double* copies_d;      // [K] comb copies per instance (exact in FP64)
  double* wsum;          // [K]
  unsigned long long* esc_fx;  // [2K] escaped energy, fixed point (units of wsum * 2^-60)
  unsigned long long* dep_fx;  // [n_cells] deposited energy, fixed point
  double* comb_after;    // [K]
  double* e_side;        // [2K]
  double* e_emit;        // [K]
  double* comb_before;   // [K]
  // workspace: per entry / per tile
  int* cnt;              // [n_slots] comb copies per entry
  long long* blk;        // [max_tiles + 1]
  unsigned long long* queue;
  // tracking launch
  int chunk, refill_min;
  int max_cells;         // largest nc_k (0: not given): the work-unit tracking stages tables in shared memory
  int form;              // imc_batch_launch.form
};

constexpr int BATCH_TILE = 1024;   // comb tile (entries per block pass)

extern unsigned long long g_imc_launches;
void imc_note_cuda_error(int e);  // imc_last_cuda_error() reports it

// imc_batch_plan.cu (no FMA contraction: counts and sums as the single-problem kernels)
cudaError_t imc_batch_launch_setup(const BatchArgs& a, const double* T0, cudaStream_t s);
cudaError_t imc_batch_launch_material_fleck(const BatchArgs& a, int update, cudaStream_t s);
cudaError_t imc_batch_launch_plan(const BatchArgs& a, cudaStream_t s);
cudaError_t imc_batch_launch_ic_plan(const BatchArgs& a, const double* tr, cudaStream_t s);
cudaError_t imc_batch_launch_prefix(const BatchArgs& a, cudaStream_t s);
cudaError_t imc_batch_launch_comb_plan(const BatchArgs& a, cudaStream_t s);
cudaError_t imc_batch_launch_ledger(const BatchArgs& a, int init, cudaStream_t s);

// imc_batch.cu
cudaError_t imc_batch_launch_fill(const BatchArgs& a, int ic, long long bound, cudaStream_t s);
cudaError_t imc_batch_launch_wsum(const BatchArgs& a, cudaStream_t s);
cudaError_t imc_batch_launch_track(const BatchArgs& a, int block, int grid, cudaStream_t s);
cudaError_t imc_batch_launch_comb_ecen(const BatchArgs& a, cudaStream_t s);
cudaError_t imc_batch_launch_comb_copy(const BatchArgs& a, cudaStream_t s);
