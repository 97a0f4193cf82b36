/* A C99 consumer of the C ABI, as a foreign-language binding sees it: the
 * header compiles as plain C, the library links by name, and the entry
 * points that need no GPU behave as documented. Exits non-zero on any
 * mismatch. */
#include <stdio.h>
#include <string.h>

#include "hydroflux_gpu.h"

static int failures = 0;
#define CHECK(cond)                                             \
  do {                                                          \
    if (!(cond)) {                                              \
      fprintf(stderr, "check failed: %s (line %d)\n", #cond, __LINE__); \
      ++failures;                                               \
    }                                                           \
  } while (0)

int main(void) {
  hf_config cfg;
  uint64_t n = 7;
  double zeros[4] = {0.0, 0.0, 0.0, 0.0};
  hf_mesh_desc mesh;
  hf_sim* sim = NULL;

  CHECK(hf_abi_version() == HF_ABI_VERSION);
  hf_config_default(&cfg);
  CHECK(cfg.cfl == 0.4 && cfg.integrator == HF_SSPRK2 && cfg.max_dt == 60.0);
  CHECK(cfg.boundaries.north.kind == HF_BC_WALL);

  CHECK(hf_kernel_launches(&n) == HF_OK && n == 0); /* nothing launched yet */
  CHECK(hf_kernel_launches(NULL) == HF_ERR_INVALID_ARG);

  CHECK(hf_sim_step(NULL, 1.0, NULL) == HF_ERR_INVALID_ARG);
  CHECK(strlen(hf_last_error()) > 0);

  /* argument checks run before any CUDA call */
  memset(&mesh, 0, sizeof mesh);
  mesh.n_rows = 2;
  mesh.n_cols = 2;
  mesh.dx = 1.0;
  mesh.dy = 1.0;
  mesh.bed = zeros;
  mesh.manning_uniform = 0.03;
  cfg.cfl = 1.5;
  CHECK(hf_sim_create(&mesh, zeros, zeros, zeros, &cfg, 0, &sim) == HF_ERR_INVALID_CONFIG);
  CHECK(sim == NULL);
  cfg.cfl = 0.4;
  mesh.n_rows = 0;
  CHECK(hf_sim_create(&mesh, zeros, zeros, zeros, &cfg, 0, &sim) == HF_ERR_SHAPE_MISMATCH);

  if (failures == 0) printf("abi consumer ok\n");
  return failures == 0 ? 0 : 1;
}
