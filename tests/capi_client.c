/* A plain C caller of libzogcu, standing in for the Zig NIF shim: it includes
 * include/zogcu.h, links the shared library and calls it with host buffers,
 * as the NIF's `new`, `pagerank` and `betweenness_unweighted` would
 * (lib/zog/.Elixir.Zog.ResourceGraph.zig:94-121, :156-170).
 *
 *   capi_client check              argument and status checks (no device needed)
 *   capi_client run EDGES d it tol PageRank and Brandes of the graph in EDGES
 *
 * EDGES is a text file: the node count on the first line, then one
 * "from to" pair per line.  `run` prints "pr <v> <score>", "bc <v> <score>"
 * (%.17g) and "iterations <n>" lines; any failing call prints its status and
 * last error and exits 1. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "zogcu.h"

static int fails = 0;

#define EXPECT(cond)                                                  \
  do {                                                                \
    if (!(cond)) {                                                    \
      fprintf(stderr, "capi_client: check failed: %s (line %d)\n", #cond, __LINE__); \
      ++fails;                                                        \
    }                                                                 \
  } while (0)

static int check(void) {
  zogcu_graph* g = NULL;
  const uint32_t from[2] = {0, 1};
  EXPECT(zogcu_abi_version() == ZOGCU_ABI_VERSION);
  EXPECT(strcmp(zogcu_status_string(ZOGCU_OK), "ok") == 0);
  EXPECT(strcmp(zogcu_status_string(ZOGCU_ERR_NODE_NOT_FOUND), "node not found") == 0);
  EXPECT(zogcu_graph_create_from_edges(3, NULL, NULL, NULL, 0, NULL) == ZOGCU_ERR_INVALID_ARGUMENT);
  EXPECT(zogcu_graph_create_from_edges(3, from, NULL, NULL, 2, &g) == ZOGCU_ERR_INVALID_ARGUMENT);
  EXPECT(g == NULL);
  EXPECT(strstr(zogcu_last_error(), "null") != NULL);
  EXPECT(zogcu_pagerank(NULL, 0.85, 10, 1e-4, NULL, NULL) == ZOGCU_ERR_INVALID_ARGUMENT);
  EXPECT(zogcu_betweenness_unweighted(NULL, NULL, NULL) == ZOGCU_ERR_INVALID_ARGUMENT);
  EXPECT(zogcu_graph_destroy(NULL) == ZOGCU_OK);
  if (fails == 0) printf("check ok\n");
  return fails ? 1 : 0;
}

static int fail(const char* what, int rc) {
  fprintf(stderr, "capi_client: %s: %s (%s)\n", what, zogcu_status_string(rc), zogcu_last_error());
  return 1;
}

static int run(const char* path, double damping, uint64_t max_iter, double tol) {
  FILE* f = fopen(path, "r");
  if (!f) {
    fprintf(stderr, "capi_client: cannot open %s\n", path);
    return 1;
  }
  unsigned long long n = 0, cap = 1024, m = 0, a, b;
  if (fscanf(f, "%llu", &n) != 1) {
    fclose(f);
    return 1;
  }
  uint32_t* from = (uint32_t*)malloc(cap * sizeof(uint32_t));
  uint32_t* to = (uint32_t*)malloc(cap * sizeof(uint32_t));
  while (fscanf(f, "%llu %llu", &a, &b) == 2) {
    if (m == cap) {
      cap *= 2;
      from = (uint32_t*)realloc(from, cap * sizeof(uint32_t));
      to = (uint32_t*)realloc(to, cap * sizeof(uint32_t));
    }
    from[m] = (uint32_t)a;
    to[m] = (uint32_t)b;
    ++m;
  }
  fclose(f);

  zogcu_graph* g = NULL;
  int rc = zogcu_graph_create_from_edges((uint32_t)n, from, to, NULL, m, &g);
  free(from);
  free(to);
  if (rc != ZOGCU_OK) return fail("zogcu_graph_create_from_edges", rc);

  uint32_t cap_nodes = 0;
  uint64_t arcs = 0;
  uint64_t live = 0;
  rc = zogcu_graph_info(g, &cap_nodes, &arcs, &live);
  if (rc != ZOGCU_OK) return fail("zogcu_graph_info", rc);

  double* pr = (double*)malloc((cap_nodes ? cap_nodes : 1) * sizeof(double));
  double* bc = (double*)malloc((cap_nodes ? cap_nodes : 1) * sizeof(double));
  zogcu_stats st;
  memset(&st, 0, sizeof st);
  rc = zogcu_pagerank(g, damping, max_iter, tol, pr, &st);
  if (rc != ZOGCU_OK) return fail("zogcu_pagerank", rc);
  printf("iterations %llu\n", (unsigned long long)st.iterations);
  rc = zogcu_betweenness_unweighted(g, bc, NULL);
  if (rc != ZOGCU_OK) return fail("zogcu_betweenness_unweighted", rc);
  for (uint32_t v = 0; v < cap_nodes; ++v) printf("pr %u %.17g\n", v, pr[v]);
  for (uint32_t v = 0; v < cap_nodes; ++v) printf("bc %u %.17g\n", v, bc[v]);
  free(pr);
  free(bc);
  rc = zogcu_graph_destroy(g);
  if (rc != ZOGCU_OK) return fail("zogcu_graph_destroy", rc);
  return 0;
}

int main(int argc, char** argv) {
  if (argc >= 2 && strcmp(argv[1], "check") == 0) return check();
  if (argc == 6 && strcmp(argv[1], "run") == 0)
    return run(argv[2], atof(argv[3]), strtoull(argv[4], NULL, 10), atof(argv[5]));
  fprintf(stderr, "usage: capi_client check | capi_client run EDGES damping max_iter tol\n");
  return 2;
}
