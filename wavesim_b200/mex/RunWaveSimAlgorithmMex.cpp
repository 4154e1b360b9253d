// MATLAB MEX shim: the reference's RunWaveSimAlgorithmMex entry point
// (called at WaveSimBase.m:145-146) forwarded to the C ABI of
// libwavesim_b200.so, so that WaveSimBase.m runs unchanged with
// opt.usemex = true.
//
//   [E, diff_energy] = RunWaveSimAlgorithmMex(N, gamma, Nwiggles, wiggles, source,
//       epsilon, k02e, roi, maxIter, energy_threshold, callbackString, callback_interval)
//
// N: 1x4 double; gamma: complex single gpuArray; wiggles: Nwiggles x 1 cell of
// structs {pxe, pye, pze, gx, gy, gz} (gpuArrays, WaveSimBase.m:303-315);
// source: Source object (properties positions, values; Source.m:18-21), already
// shifted and cropped by Simulation.exec; epsilon: single; k02e: complex single;
// roi: 2x4 double; maxIter, energy_threshold, callback_interval: double;
// callbackString: char.  E is returned as a complex single gpuArray of size N
// (E', the caller divides by gamma, WaveSimBase.m:150); diff_energy as a
// 1 x iterations double row.
//
// Build (MATLAB R2018a or later, interleaved complex API; needs MATLAB's
// headers, so it is not built in this repository's CI):
//   mex -R2018a RunWaveSimAlgorithmMex.cpp -I<repo>/include \
//       -L<repo>/wavesim_b200 -lwavesim_b200 -lmwgpu
#include <cstring>
#include <string>
#include <vector>

#include "gpu/mxGPUArray.h"
#include "mex.h"
#include "wavesim_b200.h"

namespace {

struct GpuRef {  // keeps an mxGPUArray alive for the duration of the call
  mxGPUArray const* a = nullptr;
  ~GpuRef() {
    if (a) mxGPUDestroyGPUArray(a);
  }
};

const void* device_data(const mxArray* m, std::vector<GpuRef>& keep) {
  // host arrays are copied to the GPU (MATLAB's allocator), gpuArrays are used in place
  keep.emplace_back();
  keep.back().a = mxGPUCreateFromMxArray(m);
  return mxGPUGetDataReadOnly(keep.back().a);
}

double scalar(const mxArray* m) { return mxGetScalar(m); }


void on_progress(const char* type, const double* diff_energy, int64_t n, double threshold, void*) {
  // SimulationCallback(callbackType, diff_energy, energy, energy_threshold), SimulationCallback.m:1
  mxArray* args[4];
  args[0] = mxCreateString(type);
  args[1] = mxCreateDoubleMatrix(1, (mwSize)n, mxREAL);
  std::memcpy(mxGetDoubles(args[1]), diff_energy, (size_t)n * sizeof(double));
  args[2] = mxCreateDoubleMatrix(0, 0, mxREAL);
  args[3] = mxCreateDoubleScalar(threshold);
  mexCallMATLAB(0, nullptr, 4, args, "SimulationCallback");
  for (auto* a : args) mxDestroyArray(a);
}

}  // namespace

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  if (nrhs != 12) mexErrMsgIdAndTxt("wavesim:nargin", "RunWaveSimAlgorithmMex expects 12 arguments");
  mxInitGPU();
  std::vector<GpuRef> keep;
  keep.reserve(64);

  const double* Nd = mxGetDoubles(prhs[0]);
  int64_t N[4] = {(int64_t)Nd[0], (int64_t)Nd[1], (int64_t)Nd[2], mxGetNumberOfElements(prhs[0]) > 3 ? (int64_t)Nd[3] : 1};
  const void* gamma = device_data(prhs[1], keep);
  const int64_t nw = (int64_t)scalar(prhs[2]);

  std::vector<ws_wiggle> wig((size_t)nw);
  for (int64_t w = 0; w < nw; ++w) {
    const mxArray* s = mxGetCell(prhs[3], (mwIndex)w);
    auto field = [&](const char* f) { return device_data(mxGetField(s, 0, f), keep); };
    wig[w].pxe = (const float*)field("pxe");
    wig[w].pye = (const float*)field("pye");
    wig[w].pze = (const float*)field("pze");
    wig[w].gx = (const ws_complex*)field("gx");
    wig[w].gy = (const ws_complex*)field("gy");
    wig[w].gz = (const ws_complex*)field("gz");
  }

  const mxArray* positions = mxGetProperty(prhs[4], 0, "positions");
  const mxArray* values = mxGetProperty(prhs[4], 0, "values");
  const size_t nb = mxGetNumberOfElements(values);
  std::vector<ws_source_block> blocks(nb);
  for (size_t b = 0; b < nb; ++b) {
    const double* pos = mxGetDoubles(mxGetCell(positions, (mwIndex)b));
    const mxArray* v = mxGetCell(values, (mwIndex)b);
    const mwSize nd = mxGetNumberOfDimensions(v);
    const mwSize* dims = mxGetDimensions(v);
    for (int d = 0; d < 4; ++d) {
      blocks[b].position[d] = (int64_t)pos[d];
      blocks[b].size[d] = d < (int)nd ? (int64_t)dims[d] : 1;
    }
    blocks[b].values = (const ws_complex*)device_data(v, keep);  // complex single after Simulation.exec
  }

  const float epsilon = (float)scalar(prhs[5]);
  const mxComplexSingle* k = mxGetComplexSingles(prhs[6]);
  const ws_complex k02e = {k->real, k->imag};
  const double* r = mxGetDoubles(prhs[7]);
  int64_t roi[8];
  for (int i = 0; i < 8; ++i) roi[i] = (int64_t)r[i];  // column-major 2x4, as the C ABI expects
  const int64_t max_iter = (int64_t)scalar(prhs[8]);
  const double threshold = scalar(prhs[9]);
  char cb[64] = "NoCallback";
  mxGetString(prhs[10], cb, sizeof(cb));
  const int64_t cb_interval = (int64_t)scalar(prhs[11]);

  mwSize dims[4] = {(mwSize)N[0], (mwSize)N[1], (mwSize)N[2], (mwSize)N[3]};
  mxGPUArray* E = mxGPUCreateGPUArray(4, dims, mxSINGLE_CLASS, mxCOMPLEX, MX_GPU_DO_NOT_INITIALIZE);
  std::vector<double> hist((size_t)max_iter + (size_t)nw + 1);
  int64_t n_it = 0;
  const bool want_cb = std::strcmp(cb, "NoCallback") != 0;
  const int rc = ws_run_algorithm(N, (const ws_complex*)gamma, nw, wig.data(), (int64_t)nb, blocks.data(), epsilon,
                                  k02e, roi, max_iter, threshold, cb, cb_interval, want_cb ? on_progress : nullptr,
                                  nullptr, WS_DEVICE, (ws_complex*)mxGPUGetData(E), hist.data(), &n_it);
  if (rc != WS_OK) {
    mxGPUDestroyGPUArray(E);
    mexErrMsgIdAndTxt("wavesim:b200", "RunWaveSimAlgorithmMex: %s", ws_last_error());
  }
  plhs[0] = mxGPUCreateMxArrayOnGPU(E);
  mxGPUDestroyGPUArray(E);
  if (nlhs > 1) {
    plhs[1] = mxCreateDoubleMatrix(1, (mwSize)n_it, mxREAL);
    std::memcpy(mxGetDoubles(plhs[1]), hist.data(), (size_t)n_it * sizeof(double));
  }
}
