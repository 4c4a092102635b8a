/* The user program of user_diffusion.c with its stencil written in the DSL
 * (dsl_kernels.c) and compiled by the front end: PSB_DSL_REGISTER fills a
 * psb_compiled_stencil from the kernel library and registers it, giving the
 * id PSStencilMap takes. Usage: dsl_diffusion nx ny nz count in out */
#include <stdio.h>
#include <stdlib.h>

#include "physis_b200.h"

int main(int argc, char *argv[]) {
  PSInit(&argc, &argv, 3, 0, 0, 0);
  if (argc < 7) return 2;
  int nx = atoi(argv[1]), ny = atoi(argv[2]), nz = atoi(argv[3]), count = atoi(argv[4]);
  int diffuse = 0;
  psb_status st;
  PSB_DSL_REGISTER(diffuse, &diffuse, &st);
  if (st != PSB_OK) return 4;
  size_t n = (size_t)nx * ny * nz;
  float *buf = (float *)malloc(n * sizeof(float));
  FILE *f = fopen(argv[5], "rb");
  if (!f || fread(buf, sizeof(float), n, f) != n) return 3;
  fclose(f);
  PSGrid3DFloat u = PSGrid3DFloatNew(nx, ny, nz);
  PSGrid3DFloat un = PSGrid3DFloatNew(nx, ny, nz);
  PSDomain3D dom = PSDomain3DNew(0, nx, 0, ny, 0, nz);
  float ce = 0.1f, cw = 0.1f, cn = 0.1f, cs = 0.1f, ct = 0.1f, cb = 0.1f, cc = 0.4f;
  PSGridCopyin(u, buf);
  PSStencilRun(PSStencilMap(diffuse, dom, u, un, ce, cw, cn, cs, ct, cb, cc),
               PSStencilMap(diffuse, dom, un, u, ce, cw, cn, cs, ct, cb, cc), count / 2);
  PSGridCopyout(u, buf);
  float sum = 0;
  PSReduce(&sum, PS_SUM, u);
  printf("%.9g\n", sum);
  f = fopen(argv[6], "wb");
  fwrite(buf, sizeof(float), n, f);
  fclose(f);
  PSGridFree(u);
  PSGridFree(un);
  PSFinalize();
  free(buf);
  return 0;
}
