// Batched filter bank over channels of uneven length: per channel c
//     u = FIR_valid(x_c, h_c)          (T_c taps, DSPLIB_fir semantics)
//     y = cascade of S_c DF2 biquads (u) from a zero state
// and its adjoint (gradients w.r.t. x, taps and the natural biquad
// coefficients).  Channels are packed densely: x/y at xOff[c] (length L_c;
// u and y use the first Lu_c = L_c - T_c + 1 entries), taps at hOff[c],
// coefficients [S_c][b0 b1 b2 a1 a2] at cOff[c].
//
// Kernels (every launch covers the whole batch):
//   fir_bf16x3_ragged_kernel (fir_tc.cu)  FIR forward (valid correlation) and
//                          input gradient (full convolution with the same taps)
//                          as split-BF16x3 tcgen05 contractions over runs of
//                          8192-output tiles, one run per CTA.
//   bank_tables_kernel, bank_transition_kernel, bank_unit_kernel, bank_chain_kernel,
//   bank_adjoint_kernel, bank_coef_kernel (bank_scan.cu)
//                          the cascade split along time into 512-sample units
//                          (one warp each) chained per channel through the
//                          cascade's 2S-dimensional state: unit aggregates, the
//                          chain (one state per unit and stage: the checkpoints),
//                          outputs; the adjoint the same in reverse time, with
//                          each unit's forward recomputed from the checkpoints
//                          (no stage output is stored).
//   fir_dh_bf16x3_kernel (fir_tc.cu) / fir_dh_reduce_kernel  taps gradient
//                          dh[T-1-c] = sum_j gu[j] x[j+c] as split-BF16x3
//                          tcgen05 contractions over runs of 8192-sample tiles,
//                          partial sums per run added in run order (deterministic).
//   mse_partial_kernel / mse_reduce_kernel  loss and its gradient.
//
// Work buffer (forward -> adjoint, floats): FIR output plane (sum of round16(Lu)),
// forward checkpoints, forward unit aggregates, stage tables, unit transitions.
// Scratch (adjoint): gradient w.r.t. u, adjoint aggregates and checkpoints,
// coefficient-gradient partial sums per unit and stage, taps-gradient partials
// (also the loss partials).
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <mutex>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "dsplib_internal.h"
#include "scan_common.cuh"
#include "tc_common.cuh"

namespace dsplib {

struct RaggedPlan {
   int C = 0;
   long long totalLen = 0, totalTaps = 0, totalCoefs = 0, totalOut = 0;
   long long planeStride = 0; // floats of the FIR output plane: sum of round16(Lu)
   int Smax = 0, Tmax = 0, totalStages = 0;
   int nFwdItems = 0, nFirFwdRuns = 0, nFirDxRuns = 0, nUnits = 0;
   long long nCk = 0;  // unit states (float2): sum over channels of units x stages
   long long nPhi = 0; // doubles of the unit transitions
   long long nGrp = 0; // floats of chain group states
   RaggedChan *dChan = nullptr;
   int2 *dFwdItems = nullptr;   // (channel, 2048-sample tile over Lu): taps-gradient partials, loss
   int4 *dFirFwdRuns = nullptr; // (channel, first tile, tiles): FIR forward, 8192-output tiles over Lu
   int4 *dFirDxRuns = nullptr;  // the same over L: FIR input gradient
   int *dDhStart = nullptr;     // first taps-gradient slot of each channel (C + 1 entries)
   int4 *dDhRuns = nullptr;     // (channel, first tile, tiles, slot): taps gradient, longest first
   int nDhRuns = 0;
   int2 *dUnits = nullptr;      // cascade units (channel, unit index)
   int *dChainOrder = nullptr;  // channels by unit count, most first: the chains' CTA order
   int *err = nullptr;          // error word of the tensor-core kernels (mapped page-locked)
   int device = 0;
   // work buffer layout (float offsets)
   long long wCk = 0, wAgg = 0, wTab = 0, wPhi = 0, wGrp = 0, wTotal = 0;
   // scratch layout (float offsets)
   long long sAgg = 0, sCk = 0, sGrp = 0, sPart = 0, sLoss = 0, sDh = 0, sTotal = 0;
   // host-buffer steps: the channel table, and contiguous channel segments (each with a
   // plan of its own) that are copied in, filtered and copied out as a pipeline
   std::vector<int> hLen, hTaps, hStages;
   struct Segment {
      int c0, c1;            // channels [c0, c1)
      long long x0, x1;      // samples
      long long h0, h1;      // taps
      long long k0, k1;      // coefficients
      RaggedPlan *plan;
   };
   std::vector<Segment> segs;
   // units ordered by their channel's stage count, deepest first, in buckets of one count
   std::vector<int> bucketS, bucketStart; // bucketStart has one entry more (the end)
   // auxiliary streams and events of the adjoint's bucket launches (created with the plan)
   static constexpr int kAux = 3;
   cudaStream_t aux[kAux] = {};
   cudaEvent_t fork = nullptr, join[kAux] = {};
   int nAux = 0;
   // the fork / join events are per plan: calls on one plan from several host threads
   // queue their adjoints one at a time
   std::mutex forkMu;
   long long segWork = 0, segScratch = 0; // largest work / scratch of one segment
   // device buffers of the host-buffer step (allocated by its first call, kept with the
   // plan), and whether it returns once queued (DSPLIB_gpu_raggedPlanSetAsync)
   float *hBlk = nullptr, *hWork = nullptr, *hScratch = nullptr;
   int async = 0;
};

namespace {


constexpr int kRTile = 2048; // samples per item of the taps-gradient partials and the loss
constexpr int kRaggedMaxStages = 64;

// Taps gradient: the per-run partial sums of fir_dh_bf16x3_kernel (fir_tc.cu), one
// 512-float slot per run, slots of a channel consecutive and in time order, summed in
// that order in FP64 (deterministic):  gtaps[T - 1 - c] = sum_slots part[slot][c].
constexpr int kDhMaxT = 512;
// Tiles per run of the taps gradient: each run (one CTA) pays a set-up, a first tile
// staged before any MMA and a diagonal-sum epilogue, so runs span up to 16 tiles
// (131072 samples summed in FP32 in TMEM; runs added in FP64).
constexpr int kDhRunTiles = 16;

__global__ void __launch_bounds__(256) fir_dh_reduce_kernel(const RaggedChan *chans, const int *start,
                                                             const float *part, float *gtaps)
{
   const RaggedChan c = chans[blockIdx.x];
   for (int cc = threadIdx.x; cc < c.T; cc += 256) {
      double s = 0.0;
      for (int i = start[blockIdx.x]; i < start[blockIdx.x + 1]; i++) s += part[(long long) i * kDhMaxT + cc];
      gtaps[c.hOff + c.T - 1 - cc] = (float) s;
   }
}

// Mean squared error over the valid output samples: gy = scale * (y - target)
// (scale = 2 / n), zero on each channel's T - 1 tail samples; per-item FP64
// partial sums of (y - target)^2, then one block sums them in item order.
__global__ void __launch_bounds__(256) mse_partial_kernel(const RaggedChan *chans, const int2 *items,
                                                           const float *y, const float *target, float *gy,
                                                           double *part, float scale)
{
   const int2 it = items[blockIdx.x];
   const RaggedChan c = chans[it.x];
   const int j0 = it.y * kRTile;
   const int j1 = min(j0 + kRTile, c.Lu);
   double acc = 0.0;
   for (int j = j0 + threadIdx.x; j < j1; j += 256) {
      const float d = y[c.xOff + j] - target[c.xOff + j];
      gy[c.xOff + j] = scale * d;
      acc += (double) d * d;
   }
   if (j1 == c.Lu)
      for (int j = c.Lu + threadIdx.x; j < c.L; j += 256) gy[c.xOff + j] = 0.0f;
   __shared__ double red[256];
   red[threadIdx.x] = acc;
   __syncthreads();
   for (int w = 128; w > 0; w >>= 1) {
      if ((int) threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
      __syncthreads();
   }
   if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// loss[0] = invCount * the sum of the partials (in a fixed order); with `sum`, the
// FP64 sum itself goes to sum[0] instead (one segment of a host-buffer step).
__global__ void __launch_bounds__(1024) mse_reduce_kernel(const double *part, int n, double invCount, float *loss,
                                                          double *sum)
{
   __shared__ double red[1024];
   // four independent sums per thread keep four loads in flight
   double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
   int i = threadIdx.x;
   for (; i + 3 * 1024 < n; i += 4 * 1024) {
      s0 += part[i];
      s1 += part[i + 1024];
      s2 += part[i + 2048];
      s3 += part[i + 3072];
   }
   for (; i < n; i += 1024) s0 += part[i];
   red[threadIdx.x] = (s0 + s1) + (s2 + s3);
   __syncthreads();
   for (int w = 512; w > 0; w >>= 1) {
      if ((int) threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
      __syncthreads();
   }
   if (threadIdx.x == 0) {
      if (sum)
         sum[0] = red[0];
      else
         loss[0] = (float) (red[0] * invCount);
   }
}

// The segments' sums of squares, added in segment order.
__global__ void mse_segments_kernel(const double *sums, int n, double invCount, float *loss)
{
   double s = 0.0;
   for (int i = 0; i < n; i++) s += sums[i];
   loss[0] = (float) (s * invCount);
}

template <typename T> cudaError_t upload(T **dst, const std::vector<T> &v)
{
   cudaError_t e = cudaMalloc((void **) dst, std::max<size_t>(1, v.size()) * sizeof(T));
   if (e != cudaSuccess) return e;
   if (v.empty()) return cudaSuccess;
   return cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
}

} // namespace

static void freePlan(RaggedPlan *p)
{
   if (!p) return;
   cudaFree(p->dChan);
   cudaFree(p->dFwdItems);
   cudaFree(p->dFirFwdRuns);
   cudaFree(p->dFirDxRuns);
   cudaFree(p->dDhStart);
   cudaFree(p->dDhRuns);
   cudaFree(p->dUnits);
   cudaFree(p->dChainOrder);
   freeErrorWord(p->err);
   for (RaggedPlan::Segment &g : p->segs) freePlan(g.plan);
   for (int i = 0; i < p->nAux; i++) {
      cudaStreamDestroy(p->aux[i]);
      cudaEventDestroy(p->join[i]);
   }
   if (p->fork) cudaEventDestroy(p->fork);
   cudaFree(p->hBlk);
   cudaFree(p->hWork);
   cudaFree(p->hScratch);
   delete p;
}

static long long align4(long long n) { return (n + 3) & ~3LL; }

// Makes the plan's device current for the duration of a call (and restores the
// caller's device afterwards): the plan's tables and the kernels' scratch live there.
class PlanDevice {
 public:
   explicit PlanDevice(const RaggedPlan *p)
   {
      ok_ = cudaGetDevice(&prev_) == cudaSuccess;
      if (ok_ && prev_ != p->device) {
         ok_ = cudaSetDevice(p->device) == cudaSuccess;
         switched_ = ok_;
      }
   }
   ~PlanDevice()
   {
      if (switched_) (void) cudaSetDevice(prev_);
   }
   bool ok() const { return ok_; }

 private:
   int prev_ = 0;
   bool ok_ = false, switched_ = false;
};

int raggedPlanDevice(DSPLIB_gpu_raggedPlan plan)
{
   const RaggedPlan *p = (const RaggedPlan *) plan;
   return p ? p->device : -1;
}

} // namespace dsplib

using namespace dsplib;

extern "C" {

// Plan with FIR work lists of runs of up to runTiles tiles (forward and input gradient;
// the taps gradient keeps kDhRunTiles, so its partial sums, and with them its
// rounding, do not depend on the choice).
static DSPLIB_STATUS raggedPlanBuild(DSPLIB_gpu_raggedPlan *plan, int32_t numChannels, const int32_t *length,
                                     const int32_t *taps, const int32_t *stages, int runTiles)
{
   if (!plan || !length || !taps || !stages || numChannels <= 0) return DSPLIB_ERR_NULL_POINTER;
   *plan = nullptr;
   RaggedPlan *p = new RaggedPlan();
   p->C = numChannels;
   std::vector<RaggedChan> ch(numChannels);
   std::vector<int2> fwd, units;
   std::vector<int4> firFwd, firDx, dhRuns;
   std::vector<int> start(numChannels + 1);
   // runs of up to runTiles consecutive 8192-output tiles of one channel
   auto addRuns = [runTiles](std::vector<int4> &runs, int c, int outLen) {
      const int tiles = (outLen + kFirBfTile - 1) / kFirBfTile;
      for (int t = 0; t < tiles; t += runTiles) runs.push_back(make_int4(c, t, std::min(runTiles, tiles - t), 0));
   };
   long long xo = 0, ho = 0, co = 0, po = 0, ck = 0, ph = 0, gr = 0;
   for (int c = 0; c < numChannels; c++) {
      const int L = length[c], T = taps[c], S = stages[c];
      if (T < 1 || T > kFirBfMaxTaps || L < T || S < 0 || S > kRaggedMaxStages) {
         delete p;
         return DSPLIB_ERR_INVALID_DIMENSION;
      }
      const int Lu = L - T + 1;
      const int nu = (Lu + kBankSpan - 1) / kBankSpan;
      ch[c] = RaggedChan{xo, ho, co, po, L, T, S, Lu, ck, ph, gr};
      gr += 2LL * S * ((nu + 31) / 32);
      po += (Lu + 15) & ~15;
      ck += (long long) nu * S;
      ph += bankTransitionDoubles(S);
      xo += L;
      p->totalOut += Lu;
      ho += T;
      co += 5LL * S;
      p->Smax = std::max(p->Smax, S);
      p->Tmax = std::max(p->Tmax, T);
      start[c] = (int) dhRuns.size();
      for (int t = 0; t * kRTile < Lu; t++) fwd.push_back(make_int2(c, t));
      {
         const int tiles = (Lu + kFirBfTile - 1) / kFirBfTile;
         for (int t = 0; t < tiles; t += kDhRunTiles)
            dhRuns.push_back(make_int4(c, t, std::min(kDhRunTiles, tiles - t), (int) dhRuns.size()));
      }
      for (int j = 0; j < nu; j++) units.push_back(make_int2(c, j));
      addRuns(firFwd, c, Lu);
      addRuns(firDx, c, L);
   }
   start[numChannels] = (int) dhRuns.size();
   // longest runs first, so the short ones fill in behind them
   auto longer = [](const int4 &a, const int4 &b) { return a.z > b.z; };
   std::stable_sort(firFwd.begin(), firFwd.end(), longer);
   std::stable_sort(firDx.begin(), firDx.end(), longer);
   std::stable_sort(dhRuns.begin(), dhRuns.end(), longer);
   // the chains run one CTA per channel, their time in proportion to its units: the longest
   // channels start first, so that no long chain is left for the last wave
   std::vector<int> chainOrder(numChannels);
   for (int c = 0; c < numChannels; c++) chainOrder[c] = c;
   std::stable_sort(chainOrder.begin(), chainOrder.end(), [&](int a, int b) { return ch[a].Lu > ch[b].Lu; });
   if (co / 5 > INT_MAX || units.size() > (size_t) INT_MAX) {
      delete p;
      return DSPLIB_ERR_INVALID_DIMENSION;
   }
   p->totalLen = xo;
   p->planeStride = po;
   p->totalTaps = ho;
   p->totalCoefs = co;
   p->totalStages = (int) (co / 5);
   p->nCk = ck;
   p->nPhi = ph;
   p->nGrp = gr;
   p->nFwdItems = (int) fwd.size();
   p->nFirFwdRuns = (int) firFwd.size();
   p->nFirDxRuns = (int) firDx.size();
   // deepest cascades first, one bucket per stage count: the adjoint's last pass sizes its
   // shared memory per bucket (stage sequences of S - 1 stages), so shallow cascades pack
   // more warps per SM
   std::stable_sort(units.begin(), units.end(),
                    [&](const int2 &a, const int2 &b) { return stages[a.x] > stages[b.x]; });
   for (size_t i = 0; i < units.size(); i++)
      if (i == 0 || stages[units[i].x] != stages[units[i - 1].x]) {
         p->bucketS.push_back(stages[units[i].x]);
         p->bucketStart.push_back((int) i);
      }
   p->bucketStart.push_back((int) units.size());
   p->nUnits = (int) units.size();
   p->nDhRuns = (int) dhRuns.size();
   p->hLen.assign(length, length + numChannels);
   p->hTaps.assign(taps, taps + numChannels);
   p->hStages.assign(stages, stages + numChannels);
   cudaGetDevice(&p->device);
   p->err = allocErrorWord();
   if (p->bucketS.size() > 1) {
      bool ok = cudaEventCreateWithFlags(&p->fork, cudaEventDisableTiming) == cudaSuccess;
      for (int i = 0; ok && i < RaggedPlan::kAux; i++) {
         ok = cudaStreamCreateWithFlags(&p->aux[i], cudaStreamNonBlocking) == cudaSuccess;
         if (ok && cudaEventCreateWithFlags(&p->join[i], cudaEventDisableTiming) != cudaSuccess) {
            cudaStreamDestroy(p->aux[i]);
            ok = false;
         }
         if (ok) p->nAux = i + 1;
      }
      (void) cudaGetLastError(); // without auxiliary streams the buckets run in sequence
   }
   // work buffer: u | forward checkpoints | forward aggregates | stage tables | unit transitions
   p->wCk = align4(p->planeStride);
   p->wAgg = p->wCk + align4(2 * p->nCk);
   p->wTab = p->wAgg + align4(2 * p->nCk);
   p->wPhi = p->wTab + (long long) kBankTabFloats * p->totalStages;
   p->wGrp = p->wPhi + align4(2 * p->nPhi);
   p->wTotal = p->wGrp + align4(p->nGrp);
   // scratch: g | adjoint aggregates | adjoint checkpoints | coefficient partials | taps partials
   p->sAgg = align4(p->totalLen);
   p->sCk = p->sAgg + align4(2 * p->nCk);
   p->sGrp = p->sCk + align4(2 * p->nCk);
   p->sPart = p->sGrp + align4(p->nGrp);
   p->sLoss = p->sPart + align4(5 * p->nCk);
   p->sDh = p->sLoss + align4(2LL * p->nUnits); // unit sums of squares (doubles) of the fused loss
   p->sTotal = p->sDh + align4(std::max((long long) p->nDhRuns * kDhMaxT, 2LL * p->nFwdItems));
   const bool ok = upload(&p->dChan, ch) == cudaSuccess && upload(&p->dFwdItems, fwd) == cudaSuccess &&
                   upload(&p->dFirFwdRuns, firFwd) == cudaSuccess && upload(&p->dFirDxRuns, firDx) == cudaSuccess &&
                   upload(&p->dDhStart, start) == cudaSuccess && upload(&p->dDhRuns, dhRuns) == cudaSuccess &&
                   upload(&p->dUnits, units) == cudaSuccess && upload(&p->dChainOrder, chainOrder) == cudaSuccess;
   if (!ok) {
      freePlan(p);
      return DSPLIB_ERR_FAILURE;
   }
   *plan = (DSPLIB_gpu_raggedPlan) p;
   return DSPLIB_SUCCESS;
}

// Autotuner key of a bank's FIR run length, and its candidates.
static std::string bankRunsKey(int C, const int32_t *length, const int32_t *taps)
{
   long long total = 0;
   int Tmax = 0;
   for (int c = 0; c < C; c++) {
      total += length[c];
      Tmax = std::max(Tmax, (int) taps[c]);
   }
   char buf[128];
   snprintf(buf, sizeof(buf), "bank_runs|ch=2^%d|samples=2^%d|Tmax=%d|sms=%d", tuneClass(C), tuneClass(total),
            Tmax, deviceSms());
   return buf;
}

// Time the forward FIR over scratch filled with a hashed pattern, with work lists of each candidate run
// length; the fastest is stored under key.
static void bankRunsMeasure(const RaggedPlan *p, const std::string &key)
{
   const int cands[] = {1, 2, 4, 8, 16};
   float *x = nullptr, *h = nullptr, *u = nullptr;
   std::vector<int4 *> lists;
   std::vector<int> counts;
   bool ok = cudaMalloc(&x, std::max<long long>(1, p->totalLen) * 4) == cudaSuccess &&
             cudaMalloc(&h, std::max<long long>(1, p->totalTaps) * 4) == cudaSuccess &&
             cudaMalloc(&u, std::max<long long>(1, p->planeStride) * 4) == cudaSuccess &&
             tuneFill(x, std::max<long long>(1, p->totalLen) * 4, true) &&
             tuneFill(h, std::max<long long>(1, p->totalTaps) * 4, true);
   for (int rt : cands) {
      if (!ok) break;
      std::vector<int4> runs;
      for (int c = 0; c < p->C; c++) {
         const int tiles = (p->hLen[c] - p->hTaps[c] + 1 + kFirBfTile - 1) / kFirBfTile;
         for (int t = 0; t < tiles; t += rt) runs.push_back(make_int4(c, t, std::min(rt, tiles - t), 0));
      }
      std::stable_sort(runs.begin(), runs.end(), [](const int4 &a, const int4 &b) { return a.z > b.z; });
      int4 *d = nullptr;
      ok = upload(&d, runs) == cudaSuccess;
      lists.push_back(d);
      counts.push_back((int) runs.size());
   }
   if (ok) {
      std::vector<int> cv(cands, cands + 5);
      (void) tunePick(key, cv, [&](int rt, cudaStream_t s) {
         int i = 0;
         while (cands[i] != rt) i++;
         return launchFirBf16x3Ragged(p->dChan, lists[i], counts[i], x, h, u, false, p->Tmax, p->err, s);
      });
   }
   (void) cudaGetLastError();
   for (int4 *d : lists) cudaFree(d);
   cudaFree(x);
   cudaFree(h);
   cudaFree(u);
   if (p->err) *(volatile int *) p->err = 0;
}

DSPLIB_STATUS DSPLIB_gpu_raggedPlanCreate(DSPLIB_gpu_raggedPlan *plan, int32_t numChannels, const int32_t *length,
                                          const int32_t *taps, const int32_t *stages)
{
   if (!plan || !length || !taps || !stages || numChannels <= 0) return DSPLIB_ERR_NULL_POINTER;
   const std::string key = bankRunsKey(numChannels, length, taps);
   int runTiles = kFirBfRunTiles;
   int c = 0;
   const bool cached = tuneLookup(key, &c) && c >= 1 && c <= 64;
   if (cached) runTiles = c;
   DSPLIB_STATUS st = raggedPlanBuild(plan, numChannels, length, taps, stages, runTiles);
   if (st != DSPLIB_SUCCESS || cached || tuneMode() != DSPLIB_GPU_TUNE_MEASURE) return st;
   for (int i = 0; i < numChannels; i++)
      if (taps[i] > kFirBfMaxTaps) return st;
   bankRunsMeasure((RaggedPlan *) *plan, key);
   if (tuneLookup(key, &c) && c != runTiles && c >= 1 && c <= 64) {
      DSPLIB_gpu_raggedPlan better = nullptr;
      if (raggedPlanBuild(&better, numChannels, length, taps, stages, c) == DSPLIB_SUCCESS) {
         freePlan((RaggedPlan *) *plan);
         *plan = better;
      }
   }
   return st;
}

int64_t DSPLIB_gpu_raggedPlanSize(DSPLIB_gpu_raggedPlan plan, int32_t what)
{
   RaggedPlan *p = (RaggedPlan *) plan;
   if (!p) return -1;
   switch (what) {
   case DSPLIB_GPU_RAGGED_SAMPLES: return p->totalLen;
   case DSPLIB_GPU_RAGGED_TAPS: return p->totalTaps;
   case DSPLIB_GPU_RAGGED_COEFS: return p->totalCoefs;
   case DSPLIB_GPU_RAGGED_WORK: return p->wTotal;
   case DSPLIB_GPU_RAGGED_SCRATCH: return p->sTotal;
   case DSPLIB_GPU_RAGGED_OUTPUTS: return p->totalOut;
   default: return -1;
   }
}

DSPLIB_STATUS DSPLIB_gpu_raggedPlanStatus(DSPLIB_gpu_raggedPlan plan)
{
   RaggedPlan *p = (RaggedPlan *) plan;
   if (!p) return DSPLIB_ERR_NULL_POINTER;
   bool expired = false;
   if (p->err && *(volatile int *) p->err != 0) {
      *(volatile int *) p->err = 0;
      expired = true;
   }
   for (const RaggedPlan::Segment &sg : p->segs) // the host-buffer step's segment plans
      if (sg.plan->err && *(volatile int *) sg.plan->err != 0) {
         *(volatile int *) sg.plan->err = 0;
         expired = true;
      }
   return expired ? DSPLIB_ERR_FAILURE : DSPLIB_SUCCESS;
}

DSPLIB_STATUS DSPLIB_gpu_raggedPlanSetAsync(DSPLIB_gpu_raggedPlan plan, int32_t async)
{
   RaggedPlan *p = (RaggedPlan *) plan;
   if (!p) return DSPLIB_ERR_NULL_POINTER;
   p->async = async ? 1 : 0;
   return DSPLIB_SUCCESS;
}

DSPLIB_STATUS DSPLIB_gpu_raggedPlanDestroy(DSPLIB_gpu_raggedPlan plan)
{
   freePlan((RaggedPlan *) plan);
   return DSPLIB_SUCCESS;
}

static BankLaunch bankLaunch(const RaggedPlan *p, const float *work)
{
   BankLaunch b{};
   b.chans = p->dChan;
   b.C = p->C;
   b.units = p->dUnits;
   b.chainOrder = p->dChainOrder;
   b.nUnits = p->nUnits;
   b.Smax = p->Smax;
   b.tables = work + p->wTab;
   b.phi = (const double *) (work + p->wPhi);
   b.u = work;
   b.aggF = (float2 *) (work + p->wAgg);
   b.ckptF = (float2 *) (work + p->wCk);
   b.groupF = (float *) (work + p->wGrp);
   b.bucketS = p->bucketS.data();
   b.bucketStart = p->bucketStart.data();
   b.nBuckets = (int) p->bucketS.size();
   b.aux = p->aux;
   b.nAux = p->nAux;
   b.fork = p->fork;
   b.join = p->join;
   return b;
}

DSPLIB_STATUS DSPLIB_gpu_firBiquadBatched_fwd(DSPLIB_gpu_raggedPlan plan, const float *x, const float *taps,
                                              const float *coefs, float *y, float *work, void *stream)
{
   RaggedPlan *p = (RaggedPlan *) plan;
   if (!p || !x || !taps || (!coefs && p->totalCoefs) || !y || !work) return DSPLIB_ERR_NULL_POINTER;
   PlanDevice dev(p);
   if (!dev.ok()) return DSPLIB_ERR_FAILURE;
   cudaStream_t s = (cudaStream_t) stream;
   float *u = work;
   BankLaunch b = bankLaunch(p, work);
   b.y = y;
   if (launchFirBf16x3Ragged(p->dChan, p->dFirFwdRuns, p->nFirFwdRuns, x, taps, u, false, p->Tmax, p->err, s) != cudaSuccess)
      return DSPLIB_ERR_FAILURE;
   if (launchBankTables(p->dChan, p->C, coefs, p->totalStages, p->Smax, work + p->wTab, (double *) (work + p->wPhi),
                        s) != cudaSuccess ||
       launchBankForward(b, s) != cudaSuccess)
      return DSPLIB_ERR_FAILURE;
   return DSPLIB_SUCCESS;
}

DSPLIB_STATUS DSPLIB_gpu_firBiquadBatched_bwd(DSPLIB_gpu_raggedPlan plan, const float *x, const float *taps,
                                              const float *coefs, const float *work, const float *gy, float *gx,
                                              float *gtaps, float *gcoefs, float *scratch, void *stream)
{
   RaggedPlan *p = (RaggedPlan *) plan;
   if (!p || !x || !taps || ((!coefs || !gcoefs) && p->totalCoefs) || !work || !gy || !gx || !gtaps || !scratch)
      return DSPLIB_ERR_NULL_POINTER;
   PlanDevice dev(p);
   if (!dev.ok()) return DSPLIB_ERR_FAILURE;
   cudaStream_t s = (cudaStream_t) stream;
   float *g = scratch;              // gradient w.r.t. the FIR output
   float *part = scratch + p->sDh; // per-tile taps-gradient partials
   BankLaunch b = bankLaunch(p, work);
   b.gy = gy;
   b.g = g;
   b.aggA = (float2 *) (scratch + p->sAgg);
   b.ckptA = (float2 *) (scratch + p->sCk);
   b.groupA = scratch + p->sGrp;
   b.part = scratch + p->sPart;
   b.gcoefs = gcoefs;
   {
      std::lock_guard<std::mutex> lock(p->forkMu);
      if (launchBankBackward(b, s) != cudaSuccess) return DSPLIB_ERR_FAILURE;
   }
   if (launchFirBf16x3Ragged(p->dChan, p->dFirDxRuns, p->nFirDxRuns, g, taps, gx, true, p->Tmax, p->err, s) != cudaSuccess)
      return DSPLIB_ERR_FAILURE;
   if (launchFirDhBf16x3Ragged(p->dChan, p->dDhRuns, p->nDhRuns, x, g, part, p->err, s) != cudaSuccess)
      return DSPLIB_ERR_FAILURE;
   fir_dh_reduce_kernel<<<p->C, 256, 0, s>>>(p->dChan, p->dDhStart, part, gtaps);
   countLaunch(1);
   return cudaGetLastError() == cudaSuccess ? DSPLIB_SUCCESS : DSPLIB_ERR_FAILURE;
}

} // extern "C"

namespace dsplib {

// The training step on device buffers: gy = scale (y - target); the loss goes to
// loss[0] (times invCount) or, with lossSum, as the plain FP64 sum to lossSum[0].
static DSPLIB_STATUS stepMseCore(RaggedPlan *p, const float *x, const float *taps, const float *coefs,
                                 const float *target, float *y, float *gy, float *loss, double *lossSum, float *gx,
                                 float *gtaps, float *gcoefs, float *work, float *scratch, float scale,
                                 double invCount, cudaStream_t s)
{
   float *g = scratch;
   BankLaunch b = bankLaunch(p, work);
   b.y = y;
   b.target = target;
   b.gyOut = gy;
   b.lossPart = (double *) (scratch + p->sLoss);
   b.scale = scale;
   b.aggA = (float2 *) (scratch + p->sAgg);
   // forward, loss gradient and the adjoint's first pass in one sweep over the units
   if (launchFirBf16x3Ragged(p->dChan, p->dFirFwdRuns, p->nFirFwdRuns, x, taps, work, false, p->Tmax, p->err, s) !=
           cudaSuccess ||
       launchBankTables(p->dChan, p->C, coefs, p->totalStages, p->Smax, work + p->wTab, (double *) (work + p->wPhi),
                        s) != cudaSuccess ||
       launchBankForward(b, s) != cudaSuccess)
      return DSPLIB_ERR_FAILURE;
   mse_reduce_kernel<<<1, 1024, 0, s>>>(b.lossPart, p->nUnits, invCount, loss, lossSum);
   countLaunch();
   // adjoint
   b.target = nullptr;
   b.gy = gy;
   b.g = g;
   b.ckptA = (float2 *) (scratch + p->sCk);
   b.groupA = scratch + p->sGrp;
   b.part = scratch + p->sPart;
   b.gcoefs = gcoefs;
   b.aggReady = true;
   cudaError_t be;
   {
      std::lock_guard<std::mutex> lock(p->forkMu);
      be = launchBankBackward(b, s);
   }
   if (be != cudaSuccess ||
       launchFirBf16x3Ragged(p->dChan, p->dFirDxRuns, p->nFirDxRuns, g, taps, gx, true, p->Tmax, p->err, s) != cudaSuccess ||
       launchFirDhBf16x3Ragged(p->dChan, p->dDhRuns, p->nDhRuns, x, g, scratch + p->sDh, p->err, s) != cudaSuccess)
      return DSPLIB_ERR_FAILURE;
   fir_dh_reduce_kernel<<<p->C, 256, 0, s>>>(p->dChan, p->dDhStart, scratch + p->sDh, gtaps);
   countLaunch();
   return cudaGetLastError() == cudaSuccess ? DSPLIB_SUCCESS : DSPLIB_ERR_FAILURE;
}

// Input bytes (x and target) per segment of a host-buffer step.
constexpr long long kStepSegmentBytes = 16LL << 20;
// Segments of one host-buffer step.  The step moves its bytes over PCIe in both directions
// at once; on B200 the 2048-channel bank took 15.7 ms with 8 segments and 16.3 ms with 16
// (the link, about 75 GB/s both directions together, not the pipeline's ends, bounds it).
// The pipeline's events are reused cyclically (a wait takes the event's state when queued).
constexpr int kStepMaxSegments = 8;

// Split the channels into up to kStepMaxSegments contiguous segments of about equal
// samples, each with a plan of its own (on the plan's device, which is current).
static bool buildSegments(RaggedPlan *p)
{
   if (!p->segs.empty()) return true;
   const long long bytes = 8LL * p->totalLen;
   int G = (int) std::min<long long>(kStepMaxSegments, std::max<long long>(1, (bytes + kStepSegmentBytes - 1) /
                                                                              kStepSegmentBytes));
   G = std::min(G, p->C);
   std::vector<RaggedPlan::Segment> segs;
   long long x = 0, h = 0, k = 0;
   int c = 0;
   for (int g = 0; g < G; g++) {
      RaggedPlan::Segment sg{};
      sg.c0 = c;
      sg.x0 = x;
      sg.h0 = h;
      sg.k0 = k;
      const long long goal = p->totalLen * (g + 1) / G;
      // at least one channel, and one left for each later segment
      do {
         x += p->hLen[c];
         h += p->hTaps[c];
         k += 5LL * p->hStages[c];
         c++;
      } while (c < p->C - (G - 1 - g) && x < goal);
      if (g + 1 == G)
         for (; c < p->C; c++) {
            x += p->hLen[c];
            h += p->hTaps[c];
            k += 5LL * p->hStages[c];
         }
      sg.c1 = c;
      sg.x1 = x;
      sg.h1 = h;
      sg.k1 = k;
      DSPLIB_gpu_raggedPlan sub = nullptr;
      if (DSPLIB_gpu_raggedPlanCreate(&sub, sg.c1 - sg.c0, &p->hLen[sg.c0], &p->hTaps[sg.c0], &p->hStages[sg.c0]) !=
          DSPLIB_SUCCESS) {
         for (RaggedPlan::Segment &o : segs) freePlan(o.plan);
         return false;
      }
      sg.plan = (RaggedPlan *) sub;
      segs.push_back(sg);
   }
   p->segWork = p->segScratch = 0;
   for (const RaggedPlan::Segment &sg : segs) {
      p->segWork = std::max(p->segWork, sg.plan->wTotal);
      p->segScratch = std::max(p->segScratch, sg.plan->sTotal);
   }
   p->segs = std::move(segs);
   return true;
}

// A device view of one array of a host-buffer step: the caller's pointer when it is
// device memory, else a slice of the staging block.
struct StepArray {
   const void *host;
   float *dev;
   bool staged;
};

} // namespace dsplib

extern "C" {

DSPLIB_STATUS DSPLIB_gpu_firBiquadBatched_stepMse(DSPLIB_gpu_raggedPlan plan, const float *x, const float *taps,
                                                  const float *coefs, const float *target, float *y, float *gy,
                                                  float *loss, float *gx, float *gtaps, float *gcoefs, float *work,
                                                  float *scratch, void *stream)
{
   RaggedPlan *p = (RaggedPlan *) plan;
   if (!p || !x || !taps || ((!coefs || !gcoefs) && p->totalCoefs) || !target || !y || !gy || !loss || !gx ||
       !gtaps || !work || !scratch)
      return DSPLIB_ERR_NULL_POINTER;
   if (p->totalOut <= 0) return DSPLIB_ERR_INVALID_DIMENSION;
   PlanDevice dev(p);
   if (!dev.ok()) return DSPLIB_ERR_FAILURE;
   return stepMseCore(p, x, taps, coefs, target, y, gy, loss, nullptr, gx, gtaps, gcoefs, work, scratch,
                      (float) (2.0 / (double) p->totalOut), 1.0 / (double) p->totalOut, (cudaStream_t) stream);
}

DSPLIB_STATUS DSPLIB_gpu_firBiquadBatched_stepMseHost(DSPLIB_gpu_raggedPlan plan, const float *x, const float *taps,
                                                      const float *coefs, const float *target, float *y, float *gy,
                                                      float *loss, float *gx, float *gtaps, float *gcoefs,
                                                      void *stream)
{
   RaggedPlan *p = (RaggedPlan *) plan;
   if (!p || !x || !taps || ((!coefs || !gcoefs) && p->totalCoefs) || !target || !y || !loss || !gx || !gtaps)
      return DSPLIB_ERR_NULL_POINTER;
   if (p->totalOut <= 0) return DSPLIB_ERR_INVALID_DIMENSION;
   PlanDevice dev(p);
   if (!dev.ok() || !buildSegments(p)) return DSPLIB_ERR_FAILURE;
   PipeContext *pc = pipeContext();
   if (!pc) return DSPLIB_ERR_FAILURE;
   cudaStream_t s = (cudaStream_t) stream;
   const int G = (int) p->segs.size();
   const long long nx = align4(p->totalLen), nh = align4(p->totalTaps), nk = align4(p->totalCoefs);
   // staging block: x | target | y | gy | gx | taps | gtaps | coefs | gcoefs | loss sums | loss
   StepArray arr[9] = {{x, nullptr, false},      {target, nullptr, false}, {y, nullptr, false},
                       {gy, nullptr, false},     {gx, nullptr, false},     {taps, nullptr, false},
                       {gtaps, nullptr, false},  {coefs, nullptr, false},  {gcoefs, nullptr, false}};
   const long long len[9] = {nx, nx, nx, nx, nx, nh, nh, nk, nk};
   const long long stagedFloats = 5 * nx + 2 * nh + 2 * nk + 2 * kStepMaxSegments + 4;
   if (!p->hBlk) {
      // the plan's own staging (not the thread's): calls on different plans may be in
      // flight together
      if (cudaMalloc(&p->hBlk, (size_t) stagedFloats * sizeof(float)) != cudaSuccess ||
          cudaMalloc(&p->hWork, (size_t) std::max(1LL, p->segWork) * sizeof(float)) != cudaSuccess ||
          cudaMalloc(&p->hScratch, (size_t) std::max(1LL, p->segScratch) * sizeof(float)) != cudaSuccess) {
         (void) cudaGetLastError();
         cudaFree(p->hBlk);
         cudaFree(p->hWork);
         p->hBlk = p->hWork = nullptr;
         return DSPLIB_ERR_FAILURE;
      }
   }
   float *blk = p->hBlk, *work = p->hWork, *scratch = p->hScratch;
   long long off = 0;
   for (int i = 0; i < 9; i++) {
      arr[i].staged = arr[i].host == nullptr || !isDevicePtr(arr[i].host);
      arr[i].dev = arr[i].staged ? blk + off : (float *) arr[i].host;
      off += len[i];
   }
   double *sums = (double *) (blk + off);
   float *lossDev = blk + off + 2 * kStepMaxSegments;
   const bool lossStaged = !isDevicePtr(loss);
   if (!lossStaged) lossDev = loss;
   auto h2d = [&](const StepArray &a, long long o, long long n) {
      if (!a.staged || n == 0) return cudaSuccess;
      return cudaMemcpyAsync(a.dev + o, (const float *) a.host + o, n * sizeof(float), cudaMemcpyHostToDevice, pc->in);
   };
   auto d2h = [&](const StepArray &a, long long o, long long n) {
      if (!a.staged || !a.host || n == 0) return cudaSuccess;
      return cudaMemcpyAsync((float *) a.host + o, a.dev + o, n * sizeof(float), cudaMemcpyDeviceToHost, pc->out);
   };
   cudaError_t e = cudaEventRecord(pc->start, s);
   if (e == cudaSuccess) e = cudaStreamWaitEvent(pc->in, pc->start, 0);
   if (e == cudaSuccess) e = cudaStreamWaitEvent(pc->comp, pc->start, 0);
   if (e == cudaSuccess) e = cudaStreamWaitEvent(pc->out, pc->start, 0);
   if (e != cudaSuccess) return pipeFail(nullptr, pc, e, "pipeline start");
   const float scale = (float) (2.0 / (double) p->totalOut);
   for (int g = 0; g < G; g++) {
      const RaggedPlan::Segment &sg = p->segs[g];
      const long long xo = sg.x0, xn = sg.x1 - sg.x0, ho = sg.h0, hn = sg.h1 - sg.h0, ko = sg.k0, kn = sg.k1 - sg.k0;
      if ((e = h2d(arr[0], xo, xn)) != cudaSuccess || (e = h2d(arr[1], xo, xn)) != cudaSuccess ||
          (e = h2d(arr[5], ho, hn)) != cudaSuccess || (e = h2d(arr[7], ko, kn)) != cudaSuccess ||
          (e = cudaEventRecord(pc->copied[g % kPipeMaxBlocks], pc->in)) != cudaSuccess ||
          (e = cudaStreamWaitEvent(pc->comp, pc->copied[g % kPipeMaxBlocks], 0)) != cudaSuccess)
         return pipeFail(nullptr, pc, e, "copy segment in");
      float *gyDev = arr[3].dev + xo;
      if (stepMseCore(sg.plan, arr[0].dev + xo, arr[5].dev + ho, arr[7].dev + ko, arr[1].dev + xo, arr[2].dev + xo,
                      gyDev, nullptr, sums + g, arr[4].dev + xo, arr[6].dev + ho, arr[8].dev + ko, work, scratch,
                      scale, 0.0, pc->comp) != DSPLIB_SUCCESS)
         return pipeFail(nullptr, pc, cudaErrorLaunchFailure, "segment step");
      if ((e = cudaEventRecord(pc->computed[g % kPipeMaxBlocks], pc->comp)) != cudaSuccess ||
          (e = cudaStreamWaitEvent(pc->out, pc->computed[g % kPipeMaxBlocks], 0)) != cudaSuccess ||
          (e = d2h(arr[2], xo, xn)) != cudaSuccess || (e = d2h(arr[3], xo, xn)) != cudaSuccess ||
          (e = d2h(arr[4], xo, xn)) != cudaSuccess || (e = d2h(arr[6], ho, hn)) != cudaSuccess ||
          (e = d2h(arr[8], ko, kn)) != cudaSuccess)
         return pipeFail(nullptr, pc, e, "copy segment out");
   }
   mse_segments_kernel<<<1, 1, 0, pc->comp>>>(sums, G, 1.0 / (double) p->totalOut, lossDev);
   countLaunch();
   if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaEventRecord(pc->done, pc->comp)) != cudaSuccess ||
       (e = cudaStreamWaitEvent(pc->out, pc->done, 0)) != cudaSuccess)
      return pipeFail(nullptr, pc, e, "loss");
   if (lossStaged && (e = cudaMemcpyAsync(loss, lossDev, sizeof(float), cudaMemcpyDeviceToHost, pc->out)) != cudaSuccess)
      return pipeFail(nullptr, pc, e, "copy loss");
   if ((e = cudaEventRecord(pc->done, pc->out)) != cudaSuccess || (e = cudaStreamWaitEvent(s, pc->done, 0)) != cudaSuccess)
      return pipeFail(nullptr, pc, e, "pipeline join");
   if (p->async) return DSPLIB_SUCCESS; // the caller synchronises `stream`, then DSPLIB_gpu_raggedPlanStatus
   if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return pipeFail(nullptr, pc, e, "pipeline join");
   bool expired = false;
   for (const RaggedPlan::Segment &sg : p->segs)
      if (sg.plan->err && *(volatile int *) sg.plan->err != 0) {
         *(volatile int *) sg.plan->err = 0;
         expired = true;
      }
   return expired ? DSPLIB_ERR_FAILURE : DSPLIB_SUCCESS;
}

DSPLIB_STATUS DSPLIB_gpu_raggedMseGrad(DSPLIB_gpu_raggedPlan plan, const float *y, const float *target, float *gy,
                                       float *loss, float *scratch, void *stream)
{
   RaggedPlan *p = (RaggedPlan *) plan;
   if (!p || !y || !target || !gy || !loss || !scratch) return DSPLIB_ERR_NULL_POINTER;
   if (p->totalOut <= 0) return DSPLIB_ERR_INVALID_DIMENSION;
   PlanDevice dev(p);
   if (!dev.ok()) return DSPLIB_ERR_FAILURE;
   cudaStream_t s = (cudaStream_t) stream;
   double *part = (double *) (scratch + p->sDh);
   mse_partial_kernel<<<p->nFwdItems, 256, 0, s>>>(p->dChan, p->dFwdItems, y, target, gy, part,
                                                   (float) (2.0 / (double) p->totalOut));
   mse_reduce_kernel<<<1, 1024, 0, s>>>(part, p->nFwdItems, 1.0 / (double) p->totalOut, loss, nullptr);
   countLaunch(2);
   return cudaGetLastError() == cudaSuccess ? DSPLIB_SUCCESS : DSPLIB_ERR_FAILURE;
}

} // extern "C"
