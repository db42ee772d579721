/*
 * oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * C API of the CPU restatement of CrisOptix's Conditional ReSTIR PT frame
 * loop (oracle/restir_oracle.cpp).  It is the checker for the CUDA product:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load it.  The product never links or calls it.
 */
#ifndef CRISB_ORACLE_H
#define CRISB_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#include "crisb.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_ctx oracle_ctx;

/* Scene as world-space triangle soup: tri_pos / tri_nrm hold 9 floats per
 * triangle (three corners), tri_mat one material index per triangle. */
oracle_ctx* oracle_create(const float* tri_pos, const float* tri_nrm,
                          const uint32_t* tri_mat, uint32_t num_tris,
                          const crisb_material* mats, uint32_t num_mats,
                          const crisb_emitter* emitters, uint32_t num_emitters,
                          const float* emitter_faces, uint32_t num_faces,
                          uint32_t width, uint32_t height,
                          const crisb_params* params);
void oracle_destroy(oracle_ctx* ctx);
int oracle_set_params(oracle_ctx* ctx, const crisb_params* params);
int oracle_set_threads(int n);
float oracle_scene_size(const oracle_ctx* ctx);

/* One Renderer::LaunchFrame; out_rgb is W*H*3 floats, read-modify-write. */
int oracle_render_frame(oracle_ctx* ctx, const crisb_camera* cam, float* out_rgb);
/* Same, with per-pass wall times (ms) written to pass_ms[6]. */
int oracle_render_frame_timed(oracle_ctx* ctx, const crisb_camera* cam,
                              float* out_rgb, double* pass_ms);
/* CRISB_MOTION_VECTORS input: num_pixels (= width * height) float pairs on the
 * host, copied; NULL clears */
int oracle_set_motion_vectors(oracle_ctx* ctx, const float* motion, uint32_t num_pixels);
/* textured materials: 6 corner uvs per oracle triangle, the textures and per
 * material (diffuse, specular, roughness) texture indices or -1 (NULL: none) */
int oracle_set_textures(oracle_ctx* ctx, const float* tri_uvs, uint32_t num_tris, const crisb_texture* textures,
                        uint32_t num_textures, const int32_t* material_textures);
/* the texture fetch alone: n (u, v) pairs -> n RGBA floats */
void oracle_tex_sample(const uint8_t* rgba, uint32_t width, uint32_t height, const float* uv, uint32_t n,
                       float* out);
uint64_t oracle_frame_index(const oracle_ctx* ctx);
uint32_t oracle_frame_random(const oracle_ctx* ctx);
/* Copy internal state in the crisb_*_rec layout (CRISB_BUF_* ids). */
int oracle_dump(const oracle_ctx* ctx, int buffer_id, void* dst, size_t bytes);
/* Every valid sample of the front suffix reservoirs re-traced past its
 * reconnection vertex from its seed (the loop index in flags bits 24-31):
 * *checked samples compared, *mismatched whose postReconF differs in any bit,
 * *nee_recon reconnected at their NEE vertex (not re-traceable, not compared). */
int oracle_check_post_recon(const oracle_ctx* ctx, uint32_t* checked, uint32_t* mismatched, uint32_t* nee_recon);
size_t oracle_dump_size(const oracle_ctx* ctx, int buffer_id);

/* ray k = rays[8k..8k+7] = (ox, oy, oz, tmin, dx, dy, dz, tmax) */
int oracle_trace(const oracle_ctx* ctx, const float* rays, crisb_trace_hit* hits,
                 uint32_t n, int any_hit);
int oracle_trace_bruteforce(const oracle_ctx* ctx, const float* rays,
                            crisb_trace_hit* hits, uint32_t n, int any_hit);

/* Plain path tracer (TraceCompletePath) accumulated in FP64: adds `spp`
 * frames (frame randoms from `seed`) into accum (W*H*3 doubles). */
int oracle_pt_accumulate(oracle_ctx* ctx, const crisb_camera* cam, uint32_t spp,
                         uint64_t seed, double* accum);

/* unit-level helpers for known-answer tests */
void oracle_pcg32(uint64_t initstate, uint64_t initseq, uint32_t n, uint32_t* out);
uint64_t oracle_tea64(uint32_t v0, uint32_t v1);
/* FP16 storage codecs (test hooks): binary16 bits and their value; octahedral
 * codes and their decoded unit vectors (dirs: n x 3 floats). */
void oracle_half(const float* in, uint32_t n, uint16_t* bits, float* back);
void oracle_srgb_root(const float* in, uint32_t n, float* out);
int oracle_tonemap_srgb8(const float* rgb, uint8_t* out, uint32_t num_pixels);
/* first float bit pattern b in (lo_bits, hi_bits] whose sRGB byte is below
 * that of b - 1, or 0 when the bytes never decrease there */
uint32_t oracle_srgb8_first_decrease(uint32_t lo_bits, uint32_t hi_bits);
void oracle_oct(const float* dirs, uint32_t n, uint32_t* codes, float* decoded);
void oracle_sincos(const float* phi, uint32_t n, float* s, float* c);
/* codes c whose re-encoded code c1 = encode(decode(c)) is not stable
 * (encode(decode(c1)) != c1); 0 means storing a loaded direction again never
 * moves its code */
uint64_t oracle_oct_unstable(const uint32_t* codes, uint32_t n);
int oracle_camera_data(const crisb_camera* cam, crisb_camera_data* out);
uint32_t oracle_frame_random_for(uint64_t seed, uint64_t frame_counter);

/* known-answer-test hooks: function `fn` of kat.h on n packed records, and
 * SampleEmitter over the given emitters (out: point, colour per draw) */
int oracle_kat(int fn, const void* in, uint32_t n, void* out);
int oracle_kat_emitter(const crisb_emitter* ems, uint32_t num_emitters, const float* faces,
                       const uint64_t* states, uint32_t n, float* out, uint64_t* state_out);

#ifdef __cplusplus
}
#endif

#endif
