/* A program in the shape the reference's CUDA translator emits
 * (translator/cuda_translator.cc:125-144 device function, :615-907 run
 * kernel with the domain guard and z loop, :298-529 host run loop with
 * 64x4 blocks, grid structs passed by value from g->dev), compiled against
 * this runtime's header and linked with libphysis_rt_b200 instead of
 * libphysis_rt_cuda. It uses only the drop-in entry points (__PSGridNew,
 * __PSGridCopyin/out, __PSGridFree, __PSReduceGridFloat, ...).
 * Usage: generated_diffusion nx ny nz count in.bin out.bin */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "physis_b200.h"

typedef struct {
  __PSDomain dom;
  __PSGrid *g1;
  int g1_index;
  __PSGrid *g2;
  int g2_index;
  float ce, cw, cn, cs, ct, cb, cc;
} __PSStencil_kernel;

__device__ static void kernel(const int x, const int y, const int z, __PSGrid3DFloat_dev *g1,
                              __PSGrid3DFloat_dev *g2, float ce, float cw, float cn, float cs,
                              float ct, float cb, float cc) {
  int nx = g1->dim[0], ny = g1->dim[1], nz = g1->dim[2];
  float c, w, e, n, s, b, t;
  c = g1->p0[__PSGridGetOffset3DDev(g1, x, y, z)];
  if (x == 0) w = c; else w = g1->p0[__PSGridGetOffset3DDev(g1, x - 1, y, z)];
  if (x == nx - 1) e = c; else e = g1->p0[__PSGridGetOffset3DDev(g1, x + 1, y, z)];
  if (y == 0) n = c; else n = g1->p0[__PSGridGetOffset3DDev(g1, x, y - 1, z)];
  if (y == ny - 1) s = c; else s = g1->p0[__PSGridGetOffset3DDev(g1, x, y + 1, z)];
  if (z == 0) b = c; else b = g1->p0[__PSGridGetOffset3DDev(g1, x, y, z - 1)];
  if (z == nz - 1) t = c; else t = g1->p0[__PSGridGetOffset3DDev(g1, x, y, z + 1)];
  g2->p0[__PSGridGetOffset3DDev(g2, x, y, z)] =
      cc * c + cw * w + ce * e + cs * s + cn * n + cb * b + ct * t;
}

__global__ void __PSStencilRun_kernel(__PSDomain dom, __PSGrid3DFloat_dev g1,
                                      __PSGrid3DFloat_dev g2, float ce, float cw, float cn,
                                      float cs, float ct, float cb, float cc) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x < dom.local_min[0] || x >= dom.local_max[0] || y < dom.local_min[1] ||
      y >= dom.local_max[1])
    return;
  for (int z = dom.local_min[2]; z < dom.local_max[2]; ++z)
    kernel(x, y, z, &g1, &g2, ce, cw, cn, cs, ct, cb, cc);
}

static float __PSStencilRun_0(int iter, __PSStencil_kernel s0, __PSStencil_kernel s1) {
  dim3 block(64, 4, 1);
  dim3 grid((unsigned)ceil(s0.dom.local_max[0] / 64.0), (unsigned)ceil(s0.dom.local_max[1] / 4.0), 1);
  for (int i = 0; i < iter; ++i) {
    __PSStencilRun_kernel<<<grid, block>>>(s0.dom, *(__PSGrid3DFloat_dev *)s0.g1->dev,
                                           *(__PSGrid3DFloat_dev *)s0.g2->dev, s0.ce, s0.cw,
                                           s0.cn, s0.cs, s0.ct, s0.cb, s0.cc);
    __PSStencilRun_kernel<<<grid, block>>>(s1.dom, *(__PSGrid3DFloat_dev *)s1.g1->dev,
                                           *(__PSGrid3DFloat_dev *)s1.g2->dev, s1.ce, s1.cw,
                                           s1.cn, s1.cs, s1.ct, s1.cb, s1.cc);
  }
  __PSCheckCudaError("__PSStencilRun_0");
  return 0.0f;
}

int main(int argc, char *argv[]) {
  PSInit(&argc, &argv, 3, 0, 0, 0);
  if (argc < 7) return 2;
  int nx = atoi(argv[1]), ny = atoi(argv[2]), nz = atoi(argv[3]), count = atoi(argv[4]);
  size_t n = (size_t)nx * ny * nz;
  float *buf = (float *)malloc(n * sizeof(float));
  FILE *f = fopen(argv[5], "rb");
  if (!f || fread(buf, sizeof(float), n, f) != n) return 3;
  fclose(f);
  PSVectorInt dims = {nx, ny, nz};
  __PSGrid *g1 = __PSGridNew(sizeof(float), 3, dims, NULL);
  __PSGrid *g2 = __PSGridNew(sizeof(float), 3, dims, NULL);
  __PSGridCopyin(g1, buf, NULL);
  PSDomain3D dom = PSDomain3DNew(0, nx, 0, ny, 0, nz);
  __PSStencil_kernel s0 = {dom, g1, 0, g2, 0, 0.1f, 0.1f, 0.1f, 0.1f, 0.1f, 0.1f, 0.4f};
  __PSStencil_kernel s1 = s0;
  s1.g1 = g2;
  s1.g2 = g1;
  __PSStencilRun_0(count / 2, s0, s1);
  __PSGridCopyout(g1, buf, NULL);
  float sum = 0;
  __PSReduceGridFloat(&sum, PS_SUM, g1);
  printf("%.9g\n", sum);
  f = fopen(argv[6], "wb");
  fwrite(buf, sizeof(float), n, f);
  fclose(f);
  __PSGridFree(g1, NULL);
  __PSGridFree(g2, NULL);
  PSFinalize();
  free(buf);
  return 0;
}
