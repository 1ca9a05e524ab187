/* A plain C client of include/graphene_gpu.h that needs no GPU: builds the
 * 7-point Poisson matrix of an 8x6x5 grid in 4 tiles through the host-side
 * entry points, reads back its layout, round-trips a vector through tile
 * order, parses a solver configuration and checks the error path. Prints
 * "ok" and exits 0 when every check passes. */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "graphene_gpu.h"

#define CHECK(cond)                                                \
  do {                                                             \
    if (!(cond)) {                                                 \
      fprintf(stderr, "check failed line %d: %s (%s)\n", __LINE__, \
              #cond, gr_last_error());                             \
      return 1;                                                    \
    }                                                              \
  } while (0)

int main(void) {
  gr_host_matrix* h = NULL;
  CHECK(gr_host_matrix_poisson(8, 6, 5, 4, GR_PART_RCB, GR_FLOAT32, &h) == GR_OK);
  gr_matrix_info info;
  CHECK(gr_host_matrix_get_info(h, &info) == GR_OK);
  CHECK(info.num_rows == 240);
  CHECK(info.num_tiles == 4);
  /* 7-point stencil: 6n minus two per boundary face cell. */
  CHECK(info.num_off_diag == 6 * 240 - 2 * (6 * 5 + 8 * 5 + 8 * 6));

  int32_t* r2t = malloc(sizeof(int32_t) * 240);
  CHECK(gr_host_matrix_row_to_tile(h, r2t) == GR_OK);
  int64_t counts[4] = {0, 0, 0, 0};
  for (int i = 0; i < 240; ++i) {
    CHECK(r2t[i] >= 0 && r2t[i] < 4);
    counts[r2t[i]]++;
  }
  int64_t sizes[12];
  CHECK(gr_host_matrix_tile_sizes(h, sizes) == GR_OK);
  for (int t = 0; t < 4; ++t) CHECK(sizes[3 * t] + sizes[3 * t + 1] == counts[t]);

  float nat[240], tile[240], back[240];
  for (int i = 0; i < 240; ++i) nat[i] = (float)i;
  CHECK(gr_host_matrix_decompose_vector(h, nat, tile, GR_FLOAT32) == GR_OK);
  CHECK(gr_host_matrix_compose_vector(h, tile, back, GR_FLOAT32) == GR_OK);
  CHECK(memcmp(nat, back, sizeof nat) == 0);

  char name[128], unknown[128];
  CHECK(gr_config_parse("{\"type\": \"IterativeRefinement\", // comment\n"
                        " \"extendedPrecisionType\": \"float64\", \"innerSolver\":"
                        " {\"type\": \"PBiCGStab\", \"preconditioner\": {\"type\": \"ILU\"}}}",
                        name, sizeof name, unknown, sizeof unknown) == GR_OK);
  CHECK(strstr(name, "IterativeRefinement") != NULL);
  CHECK(gr_config_parse("{\"type\": \"NoSuchSolver\"}", name, sizeof name, NULL, 0) != GR_OK);
  CHECK(strlen(gr_last_error()) > 0);

  gr_host_matrix_destroy(h);
  free(r2t);
  printf("ok\n");
  return 0;
}
