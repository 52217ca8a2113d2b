/*
 * nui_synth -- seeded synthetic RGB-D input for the tests and the benchmark.
 *
 * Analytic signed-distance scenes, camera trajectories and a Kinect-like depth/colour
 * renderer stand in for recorded sessions.  Built into its own library (libnui_synth.so),
 * not into libnui_b200.so: it is input generation, not part of the tracking path.
 */
#ifndef NUI_SYNTH_H
#define NUI_SYNTH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define NUI_SYNTH_API __attribute__((visibility("default")))
#else
#define NUI_SYNTH_API
#endif

/* ---------------------------------------------------------------- synthetic input
 * Seeded analytic scenes and trajectories standing in for recorded Kinect sessions. */
typedef struct nui_synth_scene nui_synth_scene;
enum { NUI_SYNTH_TABLETOP = 0, NUI_SYNTH_ROOM = 1 };
NUI_SYNTH_API nui_synth_scene* nui_synth_scene_create(int kind, uint64_t seed, float extent);
NUI_SYNTH_API void nui_synth_scene_destroy(nui_synth_scene* s);
NUI_SYNTH_API float nui_synth_scene_sdf(const nui_synth_scene* s, float x, float y, float z);
/* The analytic signed distance at n points (xyz: 3n floats). */
NUI_SYNTH_API void nui_synth_scene_sdf_many(const nui_synth_scene* s, const float* xyz, long n, float* out);
NUI_SYNTH_API void nui_synth_trajectory(int kind, uint64_t seed, int frame, float radius, float deg_per_frame,
                                  float* R_out, float* t_out);
NUI_SYNTH_API void nui_synth_render(const nui_synth_scene* s, const float* R, const float* t, int W, int H, float fx,
                              float fy, float cx, float cy, uint64_t noise_seed, int frame, int add_noise,
                              uint16_t* depth_mm, uint8_t* bgra);

#ifdef __cplusplus
}
#endif
#endif /* NUI_SYNTH_H */
