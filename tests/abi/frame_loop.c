/* frame_loop.c -- the reference app's init() / frameStep() through the C ABI
 * alone, in plain C99 (raycast_serialized_opencl.cpp:315-324 and 684-747:
 * the manager from a treelet file, the device buffer, then per frame the
 * analysis pass with paging and the render).
 *
 *   frame_loop <svo_path_base> <incore_bytes> <frames> <params.bin> <out_base>
 *
 * params.bin holds `frames` svo_frame_params records.  Writes
 * <out_base>.rgba (the last frame, width*height RGBA8), <out_base>.nodes and
 * <out_base>.attribs (the final incore pool) and prints one line of counts.
 * Exit status 0 on success, else the failing status code's magnitude. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "libsvo_b200.h"

static int fail(const char* what, int rc) {
  fprintf(stderr, "%s: status %d (%s)\n", what, rc, svo_last_error());
  return rc < 0 ? -rc : 1;
}

static int write_file(const char* base, const char* ext, const void* data, size_t bytes) {
  char path[4096];
  FILE* f;
  snprintf(path, sizeof path, "%s%s", base, ext);
  f = fopen(path, "wb");
  if (!f) return 0;
  if (fwrite(data, 1, bytes, f) != bytes) {
    fclose(f);
    return 0;
  }
  return fclose(f) == 0;
}

int main(int argc, char** argv) {
  svo_mm* mm = NULL;
  svo_mm_info info;
  svo_frame_params* frames;
  svo_trace_cfg cfg;
  svo_stats stats;
  uint32_t* rgba;
  svo_node* nodes;
  svo_attrib* attribs;
  unsigned long long incore;
  long n, i;
  uint32_t placed_total = 0;
  FILE* f;
  int rc;

  if (argc != 6) {
    fprintf(stderr, "usage: frame_loop svo_path_base incore_bytes frames params.bin out_base\n");
    return 2;
  }
  incore = strtoull(argv[2], NULL, 10);
  n = strtol(argv[3], NULL, 10);
  if (n <= 0) return 2;
  frames = (svo_frame_params*)malloc((size_t)n * sizeof *frames);
  f = fopen(argv[4], "rb");
  if (!frames || !f || fread(frames, sizeof *frames, (size_t)n, f) != (size_t)n) return 3;
  fclose(f);

  /* init(): the manager over the treelet file, then initClBuffer */
  rc = svo_mm_create(argv[1], incore, NULL, &mm);
  if (rc != SVO_OK) return fail("svo_mm_create", rc);
  rc = svo_mm_init_device_buffer(mm);
  if (rc != SVO_OK) return fail("svo_mm_init_device_buffer", rc);

  cfg.traversal = SVO_TRAVERSAL_TREELET;
  cfg.stack_size = 13;
  rgba = (uint32_t*)malloc((size_t)frames[n - 1].width * frames[n - 1].height * 4);
  if (!rgba) return 3;
  /* frameStep(): analysis pass (paging), then the frame into host memory */
  for (i = 0; i < n; ++i) {
    uint32_t placed = 0, visible = 0;
    rc = svo_mm_analysis_step(mm, &frames[i], 1, 0.0f, 0.0f, 13, NULL, &placed, &visible);
    if (rc != SVO_OK) return fail("svo_mm_analysis_step", rc);
    placed_total += placed;
    if (i == n - 1) {
      rc = svo_mm_render_host(mm, &frames[i], &cfg, rgba, NULL);
      if (rc != SVO_OK) return fail("svo_mm_render_host", rc);
    }
  }
  rc = svo_mm_sync(mm, NULL, &stats);
  if (rc != SVO_OK) return fail("svo_mm_sync", rc);
  rc = svo_mm_info_get(mm, &info);
  if (rc != SVO_OK) return fail("svo_mm_info_get", rc);

  nodes = (svo_node*)malloc((size_t)info.incore_nodes * sizeof *nodes);
  attribs = (svo_attrib*)malloc((size_t)info.incore_nodes * sizeof *attribs);
  if (!nodes || !attribs) return 3;
  rc = svo_mm_copy_incore(mm, 0, info.incore_nodes, nodes, attribs);
  if (rc != SVO_OK) return fail("svo_mm_copy_incore", rc);
  if (!write_file(argv[5], ".rgba", rgba, (size_t)frames[n - 1].width * frames[n - 1].height * 4) ||
      !write_file(argv[5], ".nodes", nodes, (size_t)info.incore_nodes * sizeof *nodes) ||
      !write_file(argv[5], ".attribs", attribs, (size_t)info.incore_nodes * sizeof *attribs))
    return 4;
  printf("placed %u resident %u of %u capped %u bounds %u\n", placed_total,
         info.num_slots - info.free_slots, info.num_treelets, stats.capped_rays, stats.bounds_errors);
  svo_mm_destroy(mm);
  free(nodes);
  free(attribs);
  free(rgba);
  free(frames);
  return 0;
}
