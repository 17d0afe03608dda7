// Checks sapb::fast_recip (Newton-Raphson from an FP32 seed) against the
// IEEE division 1.0/d on the GPU: prints the largest error in ulps.
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <cstdint>
#include <cstring>
#include "../../sap_warp_b200/csrc/sapb_device.cuh"

__global__ void k(const double* in, double* fast, double* ref, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    fast[i] = sapb::fast_recip(in[i]);
    ref[i] = 1.0 / in[i];
  }
}

static int64_t ulps(double a, double b) {
  int64_t ia, ib;
  memcpy(&ia, &a, 8);
  memcpy(&ib, &b, 8);
  int64_t d = ia - ib;
  return d < 0 ? -d : d;
}

int main() {
  const int n = 1 << 20;
  double *h = (double*)malloc(n * 8), *f = (double*)malloc(n * 8), *r = (double*)malloc(n * 8);
  srand(12345);
  for (int i = 0; i < n; ++i) {
    double u = (double)rand() / RAND_MAX, s = (rand() & 1) ? 1.0 : -1.0;
    h[i] = s * pow(10.0, -35.0 + 70.0 * u);  // spans the fast range and both fallbacks
  }
  double *dh, *df, *dr;
  cudaMalloc(&dh, n * 8);
  cudaMalloc(&df, n * 8);
  cudaMalloc(&dr, n * 8);
  cudaMemcpy(dh, h, n * 8, cudaMemcpyHostToDevice);
  k<<<(n + 255) / 256, 256>>>(dh, df, dr, n);
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) { printf("cuda error %s\n", cudaGetErrorString(e)); return 2; }
  cudaMemcpy(f, df, n * 8, cudaMemcpyDeviceToHost);
  cudaMemcpy(r, dr, n * 8, cudaMemcpyDeviceToHost);
  int64_t worst = 0;
  for (int i = 0; i < n; ++i) { int64_t u = ulps(f[i], r[i]); if (u > worst) worst = u; }
  printf("max_ulps %lld\n", (long long)worst);
  return 0;
}
