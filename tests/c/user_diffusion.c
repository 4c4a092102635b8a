/* A user program written against the translator-free C API: the shape of
 * examples/diffusion-benchmark/diffusion3d_physis.c:53-76 with the stencil
 * named by PSB_KERNEL_DIFFUSION7 instead of a C function. Reads a float
 * field, runs `count` double-buffered steps, writes the field and prints
 * PSReduce(PS_SUM). Usage: user_diffusion nx ny nz count in.bin out.bin */
#include <stdio.h>
#include <stdlib.h>

#include "physis_b200.h"

int main(int argc, char *argv[]) {
  PSInit(&argc, &argv, 3, 0, 0, 0);
  if (argc < 7) return 2;
  int nx = atoi(argv[1]), ny = atoi(argv[2]), nz = atoi(argv[3]), count = atoi(argv[4]);
  size_t n = (size_t)nx * ny * nz;
  float *buf = (float *)malloc(n * sizeof(float));
  FILE *f = fopen(argv[5], "rb");
  if (!f || fread(buf, sizeof(float), n, f) != n) return 3;
  fclose(f);
  PSGrid3DFloat f1g = PSGrid3DFloatNew(nx, ny, nz);
  PSGrid3DFloat f2g = PSGrid3DFloatNew(nx, ny, nz);
  PSDomain3D dom = PSDomain3DNew(0, nx, 0, ny, 0, nz);
  float ce = 0.1f, cw = 0.1f, cn = 0.1f, cs = 0.1f, ct = 0.1f, cb = 0.1f, cc = 0.4f;
  PSGridCopyin(f1g, buf);
  PSStencilRun(PSStencilMap(PSB_KERNEL_DIFFUSION7, dom, f1g, f2g, ce, cw, cn, cs, ct, cb, cc),
               PSStencilMap(PSB_KERNEL_DIFFUSION7, dom, f2g, f1g, ce, cw, cn, cs, ct, cb, cc),
               count / 2);
  PSGridCopyout(f1g, buf);
  float sum = 0;
  PSReduce(&sum, PS_SUM, f1g);
  printf("%.9g\n", sum);
  f = fopen(argv[6], "wb");
  fwrite(buf, sizeof(float), n, f);
  fclose(f);
  PSGridFree(f1g);
  PSGridFree(f2g);
  PSFinalize();
  free(buf);
  return 0;
}
