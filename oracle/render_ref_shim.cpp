/*
 * TEST INFRASTRUCTURE ONLY.  C entry points over the reference's own CPU
 * splatting renderer (Particle_renderer/particle_renderer/particle_renderer/
 * shadow.cpp compute_shadows, render.cpp render_smoke, write_sgi.cpp
 * write_sgi), so that tests can run the reference itself on the same inputs
 * as the CUDA renderer.  oracle/Makefile (target `ref`) compiles this file
 * together with those reference sources, read where they lie, into
 * oracle/_ref/librender_ref.so.  Nothing in the product links it.
 */
#include <cstdio>
#include <cstring>

#include "render.h"
#include "shadow.h"
#include "write_sgi.h"

static Array1<Vec3f> vec3_array(int n, const float *xyz) {
    Array1<Vec3f> x(n);
    for (int i = 0; i < n; i++) x[i] = Vec3f(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
    return x;
}

static Array1<float> float_array(int n, const float *v) {
    Array1<float> a(n);
    for (int i = 0; i < n; i++) a[i] = v[i];
    return a;
}

/* compute_shadows on n points (xyz packed), per-point density dens.  Returns
 * 1 on success (0 when the reference refuses: light too close).  illum[n]
 * receives the per-point illumination; *npix the shadow-map edge; shadow
 * (npix^2 floats, i-fastest) is written when npix^2 <= cap. */
extern "C" int ref_compute_shadows(int n, const float *xyz, float radius, float opacity, const float *dens,
                                   const float light[3], float quality, float *illum, int *npix, float *shadow,
                                   long cap) {
    Array1<Vec3f> x = vec3_array(n, xyz);
    Array1<float> d = float_array(n, dens);
    Array1<float> il;
    Array2f sm;
    const bool ok = compute_shadows(x, radius, opacity, d, Vec3f(light[0], light[1], light[2]), quality, il, sm);
    if (!ok) return 0;
    for (int i = 0; i < n; i++) illum[i] = il[i];
    *npix = sm.ni;
    if ((long)sm.ni * sm.nj <= cap)
        for (int j = 0; j < sm.nj; j++)
            for (int i = 0; i < sm.ni; i++) shadow[i + (long)sm.ni * j] = sm(i, j);
    return 1;
}

/* render_smoke into an ni x nj RGB image (image[3 * (i + ni * j) + c]). */
extern "C" void ref_render_smoke(int n, const float *xyz, const float *illum, const float *base_rgb,
                                 const float *lit_rgb, float radius, float opacity, const float *den,
                                 const float light[3], const float background[3], const float camera[3],
                                 const float target[3], float perspective, int ni, int nj, float *image) {
    Array1<Vec3f> x = vec3_array(n, xyz), base = vec3_array(n, base_rgb), lit = vec3_array(n, lit_rgb);
    Array1<float> il = float_array(n, illum), d = float_array(n, den);
    Array2<Vec3f> img(ni, nj);
    render_smoke(x, il, base, lit, radius, opacity, d, Vec3f(light[0], light[1], light[2]),
                 Vec3f(background[0], background[1], background[2]), Vec3f(camera[0], camera[1], camera[2]),
                 Vec3f(target[0], target[1], target[2]), perspective, img);
    for (int j = 0; j < nj; j++)
        for (int i = 0; i < ni; i++)
            for (int c = 0; c < 3; c++) image[3 * (i + (long)ni * j) + c] = img(i, j)[c];
}

/* write_sgi of a monochrome (channels 1) or RGB (channels 3) image. */
extern "C" int ref_write_sgi(const char *path, int ni, int nj, int channels, const float *pix, int high_precision) {
    if (channels == 1) {
        Array2f img(ni, nj);
        for (int j = 0; j < nj; j++)
            for (int i = 0; i < ni; i++) img(i, j) = pix[i + (long)ni * j];
        return write_sgi(img, high_precision != 0, "%s", path) ? 1 : 0;
    }
    Array2<Vec3f> img(ni, nj);
    for (int j = 0; j < nj; j++)
        for (int i = 0; i < ni; i++) {
            const float *p = pix + 3 * (i + (long)ni * j);
            img(i, j) = Vec3f(p[0], p[1], p[2]);
        }
    return write_sgi(img, high_precision != 0, "%s", path) ? 1 : 0;
}
