/*
 * A plain-C caller of libbnb's C ABI (include/bnb.h), as BLaDE's C++ step
 * loop would link it: no Python, no torch.
 *   abi_calls            argument and call-order checks, no device work
 *   abi_calls IN OUT     one direct-space evaluation of the system in IN
 *
 * IN (binary, little endian): int N, int nTypes, int nExcl; float box[3];
 * bnb_params; float xyz[3N]; bnb_nbond nbonds[N]; bnb_vdw vdw[nTypes^2];
 * int excl[2*nExcl].  OUT: double force64[3N], double energy64.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cuda_runtime.h>

#include "bnb.h"

#define CHECK(x, want)                                                            \
  do {                                                                            \
    int rc_ = (x);                                                                \
    if (rc_ != (want)) {                                                          \
      fprintf(stderr, "%s:%d: %s returned %d, expected %d\n", __FILE__, __LINE__, \
              #x, rc_, (want));                                                   \
      return 1;                                                                   \
    }                                                                             \
  } while (0)

static int argument_checks(void) {
  bnb_params p;
  bnb_handle *h = NULL;
  int counts[1] = {0};
  float box[3] = {40.f, 40.f, 40.f};
  bnb_outputs out;
  bnb_constraints empty;
  double x[9] = {0};
  bnb_default_params(&p);
  CHECK(bnb_create(NULL, 1, counts, &h), BNB_ERR_ARG);
  CHECK(bnb_create(&p, 0, counts, &h), BNB_ERR_ARG);
  CHECK(bnb_create(&p, 1, counts, &h), BNB_OK);
  memset(&out, 0, sizeof(out));
  CHECK(bnb_rebuild(h, NULL, box, NULL, 0), BNB_ERR_STATE);          /* before the topology */
  CHECK(bnb_compute(h, NULL, NULL, box, 1, &out, NULL), BNB_ERR_STATE);
  CHECK(bnb_set_pme(h, 5, 1.0f, NULL, box), BNB_ERR_ARG);           /* orders 4, 6, 8 */
  CHECK(bnb_set_pme(h, 6, 1.0f, NULL, box), BNB_ERR_STATE);
  CHECK(bnb_set_tuning(h, 0, 0, 2), BNB_ERR_ARG);                    /* 1..32 tiles per work item */
  CHECK(bnb_set_tuning(h, 4, 3, 9), BNB_ERR_ARG);                    /* tail 0..8 */
  CHECK(bnb_set_tuning(h, 4, 3, 0), BNB_OK);
  CHECK(bnb_destroy(h), BNB_OK);
  memset(&empty, 0, sizeof(empty));
  CHECK(bnb_holonomic_position(&empty, x, x, NULL, x, 0.02, 1e-10, 10, NULL, NULL, NULL), BNB_OK);
  CHECK(bnb_holonomic_position(NULL, x, x, NULL, x, 0.02, 1e-10, 10, NULL, NULL, NULL), BNB_ERR_ARG);
  printf("abi checks ok (%s)\n", bnb_version());
  return 0;
}

static int read_all(FILE *f, void *dst, size_t bytes) { return fread(dst, 1, bytes, f) == bytes ? 0 : 1; }

static int evaluate(const char *in, const char *outPath) {
  FILE *f = fopen(in, "rb");
  int N, nTypes, nExcl;
  float box[3];
  bnb_params p;
  if (!f || read_all(f, &N, 4) || read_all(f, &nTypes, 4) || read_all(f, &nExcl, 4) || read_all(f, box, 12) ||
      read_all(f, &p, sizeof(p)))
    return 2;
  float *xyz = malloc(sizeof(float) * 3 * N);
  bnb_nbond *nb = malloc(sizeof(bnb_nbond) * N);
  bnb_vdw *vdw = malloc(sizeof(bnb_vdw) * nTypes * nTypes);
  int *excl = malloc(sizeof(int) * 2 * (nExcl > 0 ? nExcl : 1));
  if (read_all(f, xyz, sizeof(float) * 3 * N) || read_all(f, nb, sizeof(bnb_nbond) * N) ||
      read_all(f, vdw, sizeof(bnb_vdw) * nTypes * nTypes) || read_all(f, excl, sizeof(int) * 2 * nExcl))
    return 2;
  fclose(f);

  bnb_handle *h = NULL;
  int one = 1;
  CHECK(bnb_create(&p, 1, &N, &h), BNB_OK);
  CHECK(bnb_set_topology(h, nb, &nTypes, vdw, &one, nExcl, excl, NULL), BNB_OK);
  float *pos_d;
  double *f64_d, *e64_d;
  if (cudaMalloc((void **)&pos_d, sizeof(float) * 3 * N) != cudaSuccess ||
      cudaMalloc((void **)&f64_d, sizeof(double) * 3 * N) != cudaSuccess ||
      cudaMalloc((void **)&e64_d, sizeof(double)) != cudaSuccess)
    return 3;
  cudaMemcpy(pos_d, xyz, sizeof(float) * 3 * N, cudaMemcpyHostToDevice);
  CHECK(bnb_rebuild(h, pos_d, box, NULL, 0), BNB_OK);              /* Domdec::reset_domdec */
  bnb_outputs o;
  memset(&o, 0, sizeof(o));
  o.force64 = f64_d;
  o.energy64 = e64_d;
  CHECK(bnb_compute(h, pos_d, NULL, box, 1, &o, NULL), BNB_OK);     /* getforce_nbdirect */
  if (cudaDeviceSynchronize() != cudaSuccess) return 3;
  double *f64 = malloc(sizeof(double) * 3 * N);
  double e64;
  cudaMemcpy(f64, f64_d, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost);
  cudaMemcpy(&e64, e64_d, sizeof(double), cudaMemcpyDeviceToHost);
  int status = -1;
  CHECK(bnb_status(h, NULL, 0, &status), BNB_OK);
  if (status != 0) return 4;
  CHECK(bnb_destroy(h), BNB_OK);
  FILE *g = fopen(outPath, "wb");
  if (!g) return 2;
  fwrite(f64, sizeof(double), 3 * (size_t)N, g);
  fwrite(&e64, sizeof(double), 1, g);
  fclose(g);
  cudaFree(pos_d);
  cudaFree(f64_d);
  cudaFree(e64_d);
  free(xyz); free(nb); free(vdw); free(excl); free(f64);
  printf("evaluated %d atoms, energy %.9f\n", N, e64);
  return 0;
}

int main(int argc, char **argv) {
  if (argc == 3) return evaluate(argv[1], argv[2]);
  return argument_checks();
}
