/* Oracle (test infrastructure only): CPU restatement of Shinobi's grid
 * build, DDA traversal and ray generation.  Used as the checker by the
 * tests, the smoke check and the bench's CPU baseline; never by the product. */
#ifndef SHINOBI_ORACLE_H
#define SHINOBI_ORACLE_H
#include <stdint.h>

typedef struct orc_grid orc_grid;

void orc_bounds(const float* vtx, const uint32_t* idx, uint32_t nt, float out[6]);
void orc_resolution(uint32_t nt, const float bounds[6], float lambda, int divisor, int min_res,
                    int out[3]);
orc_grid* orc_build_uniform(const float* vtx, uint32_t nv, const uint32_t* idx, uint32_t nt,
                            const float bounds[6], const int res[3]);
orc_grid* orc_build_two_level(const float* vtx, uint32_t nv, const uint32_t* idx, uint32_t nt,
                              const float bounds[6], const int res[3], float lambda_leaf,
                              uint32_t leaf_threshold);
void orc_sah_window(uint32_t nt, const float bounds[6], float lambda, float wlo, float whi, int rmin[3],
                    int rmax[3]);
uint64_t orc_sah_refs(const float* vtx, const uint32_t* idx, uint32_t nt, const float bounds[6], const int res[3]);
float orc_sah_cost(const float bounds[6], const int res[3], uint64_t refs);
void orc_sah_resolution(const float* vtx, const uint32_t* idx, uint32_t nt, const float bounds[6], float lambda,
                        float wlo, float whi, int res_out[3], float* cost_out, uint64_t* refs_out,
                        uint64_t* counts);
orc_grid* orc_build_uniform_ex(const float* vtx, uint32_t nv, const uint32_t* idx, uint32_t nt,
                               const float bounds[6], const int res[3], int insertion);
orc_grid* orc_build_two_level_ex(const float* vtx, uint32_t nv, const uint32_t* idx, uint32_t nt,
                                 const float bounds[6], const int res[3], float lambda_leaf,
                                 uint32_t leaf_threshold, int insertion);
orc_grid* orc_grid_from_arrays(int kind, const float bounds[6], const int res[3],
                               const uint32_t* cells, const uint32_t* leaves, uint64_t nleaves,
                               const uint32_t* indices, uint64_t nrefs, const float* vtx,
                               uint32_t nv, const uint32_t* idx, uint32_t nt);
void orc_grid_free(orc_grid* g);
void orc_set_reference_arithmetic(int flags);
void orc_leaf_res_reference(const orc_grid* G, float lambda, uint32_t threshold, uint32_t* out);
void orc_grid_info(const orc_grid* g, uint64_t out[8]);
const uint32_t* orc_grid_cells(const orc_grid* g);
const uint32_t* orc_grid_leaves(const orc_grid* g);
const uint32_t* orc_grid_indices(const orc_grid* g);
const uint64_t* orc_grid_top_pairs(const orc_grid* g);

int orc_num_threads(void);
void orc_set_threads(int n);
void orc_trace_closest(const orc_grid* g, const float* ox, const float* oy, const float* oz,
                       const float* dx, const float* dy, const float* dz, const float* tmax,
                       uint32_t n, uint32_t* tri, float* t, float* u, float* v, uint64_t* stats);
void orc_trace_any(const orc_grid* g, const float* ox, const float* oy, const float* oz,
                   const float* dx, const float* dy, const float* dz, const float* tmax, uint32_t n,
                   uint8_t* occluded, uint64_t* stats);
void orc_trace_brute(const float* vtx, const uint32_t* idx, uint32_t nt, const float* ox,
                     const float* oy, const float* oz, const float* dx, const float* dy,
                     const float* dz, uint32_t n, uint32_t* tri, float* t);
void orc_t_fp64(const float* vtx, const uint32_t* idx, const uint32_t* tri, const float* ox,
                const float* oy, const float* oz, const float* dx, const float* dy, const float* dz,
                uint32_t n, double* t64);

void orc_sincos_2pi(const float* u, uint32_t n, float* s, float* c);
void orc_cosine_local(const float* u1, const float* u2, uint32_t n, float* out);
void orc_philox(const uint32_t* ctr, uint32_t n, uint32_t k0, uint32_t k1, uint32_t* out);
void orc_camera(const float eye[3], const float fwd[3], const float up[3], float fov_deg,
                uint32_t resx, uint32_t resy, float out[9]);
void orc_primary_rays(const float cam[9], uint32_t resx, uint32_t resy, uint32_t image_id,
                      float* dx, float* dy, float* dz);
uint32_t orc_ao_rays(const float* vtx, const uint32_t* idx, const float* ox, const float* oy,
                     const float* oz, const float* dx, const float* dy, const float* dz,
                     const uint32_t* tri, const float* t, uint32_t n, uint32_t spp, uint32_t seed,
                     float offset, float* rox, float* roy, float* roz, float* rdx, float* rdy,
                     float* rdz, uint32_t* rpix, const uint32_t* pix);
uint32_t orc_direct_rays(const float* ox, const float* oy, const float* oz, const float* dx,
                         const float* dy, const float* dz, const uint32_t* tri, const float* t,
                         uint32_t n, uint32_t spp, uint32_t seed, uint32_t image_id,
                         const float* light15, float* rox, float* roy, float* roz, float* rdx,
                         float* rdy, float* rdz, uint32_t* rpix, const uint32_t* pix);
void orc_shade_direct(const float* vtx, const uint32_t* idx, const float* ox, const float* oy,
                      const float* oz, const float* dx, const float* dy, const float* dz,
                      const uint32_t* tri, const float* t, uint32_t n, uint32_t spp, uint32_t seed,
                      uint32_t image_id, const float* light15, const uint32_t* tri_mat,
                      const float* diffuse, uint32_t nmat, const float* ddef, const float* bg,
                      const uint8_t* occ, float* frame, float* fin, const uint32_t* pix);
void orc_pt_render(const orc_grid* g, const float cam9[9], const float eye[3], uint32_t resx,
                   uint32_t resy, uint32_t spp, uint32_t max_depth, uint32_t rr_depth, float albedo,
                   const float lpos[3], const float le1[3], const float le2[3], const float lrad[3],
                   const float bg[3], float offset, uint32_t seed, float* image);
void orc_pt_render_pixels(const orc_grid* G, const float cam9[9], const float eye[3], uint32_t resx,
                          uint32_t resy, uint32_t spp, uint32_t max_depth, uint32_t rr_depth, float albedo,
                          const float lpos[3], const float le1[3], const float le2[3], const float lrad[3],
                          const float bg[3], float offset, uint32_t seed, const uint32_t* pix,
                          uint32_t npix_sel, float* image);
uint32_t orc_compact(const uint32_t* flags, uint32_t n, uint32_t* out);

#endif
