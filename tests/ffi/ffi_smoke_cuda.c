/*
 * C smoke test of the drop-in ABI: exercises the gsplat.h v0.1 contract
 * (version, bad render mode, bad camera, PLY load, render, stats) and the
 * additive readback of gsplat_cuda.h, linking against libgsplat_ffi_c.so.
 * Exit codes: 0 ok, 3 context creation failed (e.g. no GPU), other = a
 * contract violation.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "gsplat.h"
#include "gsplat_cuda.h"

int main(int argc, char **argv) {
  const char *dataset = argc > 1 ? argv[1] : "tests/golden/minimal_ascii.ply";
  if (gsplat_version_major() != 0 || gsplat_version_minor() != 1) return 2;

  GsplatConfig bad = gsplat_config_default();
  bad.mode = 1;
  GsplatContext *ctx = (GsplatContext *)0x1;
  if (gsplat_context_create(bad, &ctx) != GSPLAT_ERROR_INVALID_ARGUMENT || ctx != NULL) return 8;

  GsplatConfig cfg = gsplat_config_default();
  cfg.width = 64;
  cfg.height = 64;
  int32_t rc = gsplat_context_create(cfg, &ctx);
  if (rc != GSPLAT_OK || ctx == NULL) {
    fprintf(stderr, "create failed: %s (%d): %s\n", gsplat_error_message(rc), rc,
            gsplat_last_error_message());
    return 3;
  }
  GsplatCamera cam = gsplat_camera_default();
  GsplatCamera badcam = cam;
  badcam.near_plane = 10.0f;
  badcam.far_plane = 1.0f;
  if (gsplat_context_set_camera(ctx, badcam) != GSPLAT_ERROR_INVALID_ARGUMENT) return 9;
  if (gsplat_context_render_frame(ctx) != GSPLAT_ERROR_SCENE_NOT_LOADED) return 10;
  if (gsplat_context_set_camera(ctx, cam) != GSPLAT_OK) return 4;
  if (gsplat_context_load_scene_path(ctx, "/nonexistent/scene.ply") != GSPLAT_ERROR_NOT_FOUND) return 11;
  if (gsplat_context_load_scene_path(ctx, dataset) != GSPLAT_OK) {
    fprintf(stderr, "load failed: %s\n", gsplat_last_error_message());
    return 5;
  }
  if (gsplat_context_render_frame(ctx) != GSPLAT_OK) {
    fprintf(stderr, "render failed: %s\n", gsplat_last_error_message());
    return 6;
  }
  GsplatStats st;
  memset(&st, 0, sizeof(st));
  if (gsplat_context_get_stats(ctx, &st) != GSPLAT_OK) return 7;
  if (st.visible_count != 2 || st.drawn_count != 2) return 12;
  unsigned char *img = (unsigned char *)malloc(64 * 64 * 4);
  if (gsplat_context_readback_rgba8(ctx, img, 64 * 64 * 4) != GSPLAT_OK) return 13;
  unsigned long long sum[4] = {0, 0, 0, 0};
  for (int i = 0; i < 64 * 64; ++i)
    for (int c = 0; c < 4; ++c) sum[c] += img[4 * i + c];
  free(img);
  printf("ffi smoke ok visible=%u drawn=%u frame_ms=%.4f means=%.4f %.4f %.4f %.4f\n",
         st.visible_count, st.drawn_count, st.frame_ms, sum[0] / (64.0 * 64 * 255),
         sum[1] / (64.0 * 64 * 255), sum[2] / (64.0 * 64 * 255), sum[3] / (64.0 * 64 * 255));
  gsplat_context_destroy(ctx);
  gsplat_context_destroy(NULL);
  return 0;
}
