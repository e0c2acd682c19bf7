/*
 * pe_oracle.c — TEST INFRASTRUCTURE (oracle): a plain-C restatement of the reference's
 * path-tracing hot path for the plain Cornell workload (Lambert surfaces, emissive triangles,
 * no environment).  Not part of the product: only tests/ load the library built from it.
 * It is pinned against the reference itself (oracle/_ref/libphoton_ref.so) by
 * tests/test_oracle_restatement.py, and then serves as a second, independent checker.
 *
 * Every routine follows the reference file:line given beside it and keeps its float operation
 * order (compiled with -ffp-contract=off), so it reproduces the reference's floats:
 *   Owen-scrambled Sobol (Burley 2020)   src/samplers/sobol_sampler.cpp:62-146 (the definition
 *                                        form of tests/test_sobol.cpp:141-175: rev ∘ LK ∘ rev)
 *   pinhole camera ray, box filter       src/engine/renderer.cpp:139-160, perspective_camera.cpp:36-40,
 *                                        pixel_filter.cpp:84-86
 *   vertex normals                       src/geometry/mesh.cpp:30-55
 *   Möller–Trumbore + hit record         src/geometry/bvh.cpp:302-316, triangle.cpp:54-100
 *   spawn offsets / shadow ray           src/geometry/ray_spawn.h:25-87, path_tracer.cpp:144-157
 *   Lambertian                           src/materials/lambertian.cpp:8-62
 *   triangle light, importance          src/lights/area_light.cpp:206-254
 *   exhaustive light selection           src/lights/light_sampler.cpp:150-241
 *   estimator (emission MIS, NEE, RR)    src/integrators/path_tracer.cpp:321-890
 *   film accumulation                    src/core/image/film.cpp:56-69
 * Intersection here is brute force (every triangle, index order, last equal hit wins), so it
 * does not depend on any acceleration structure; equal-distance ties may resolve differently
 * from the reference's BVH order.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct { float x, y, z; } v3;

static v3 mk(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static v3 add(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3 sub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3 mulv(v3 a, v3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
static v3 muls(v3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
static v3 divs(v3 a, float s) { float inv = 1.0f / s; return mk(a.x * inv, a.y * inv, a.z * inv); }
static v3 neg(v3 a) { return mk(-a.x, -a.y, -a.z); }
static float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static v3 cross(v3 a, v3 b) { return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static float len2(v3 a) { return dot(a, a); }
static v3 normalize(v3 a) { float l = sqrtf(len2(a)); return l <= 1e-20f ? mk(0, 0, 0) : divs(a, l); }
static float fmax2(float a, float b) { return (a < b) ? b : a; } /* std::max */
static float fmin2(float a, float b) { return (b < a) ? b : a; } /* std::min */
static v3 vabs(v3 a) { return mk(fabsf(a.x), fabsf(a.y), fabsf(a.z)); }
static float maxc(v3 a) { return fmax2(fmax2(a.x, a.y), a.z); }
static int finite1(float x) { uint32_t u; memcpy(&u, &x, 4); return (u & 0x7f800000u) != 0x7f800000u; }
static int finite3(v3 a) { return finite1(a.x) && finite1(a.y) && finite1(a.z); }
static int black(v3 a) { return a.x == 0.0f && a.y == 0.0f && a.z == 0.0f; }
static float lum(v3 c) { return 0.212671f * c.x + 0.715160f * c.y + 0.072169f * c.z; }
static const float PI = 3.14159265358979323846f;

/* ---- Owen-scrambled Sobol, definition form ---------------------------------------------- */
static uint32_t rev(uint32_t x) {
    x = ((x >> 1) & 0x55555555u) | ((x & 0x55555555u) << 1);
    x = ((x >> 2) & 0x33333333u) | ((x & 0x33333333u) << 2);
    x = ((x >> 4) & 0x0F0F0F0Fu) | ((x & 0x0F0F0F0Fu) << 4);
    x = ((x >> 8) & 0x00FF00FFu) | ((x & 0x00FF00FFu) << 8);
    return (x >> 16) | (x << 16);
}
static uint32_t sobol1(uint32_t i) {
    uint32_t r = 0;
    for (uint32_t v = 0x80000000u; i != 0; i >>= 1, v ^= v >> 1)
        if (i & 1u) r ^= v;
    return r;
}
static uint32_t lk(uint32_t x, uint32_t s) {
    x += s;
    x ^= x * 0x6c50b47cu;
    x ^= x * 0xb82f1e52u;
    x ^= x * 0xc7afe638u;
    x ^= x * 0x8d22f6e6u;
    return x;
}
static uint32_t nus(uint32_t x, uint32_t s) { return rev(lk(rev(x), s)); }
static uint32_t mix(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
static uint32_t hcomb(uint32_t h, uint32_t v) { return mix(h ^ (v + 0x9e3779b9u + (h << 6) + (h >> 2))); }
static float unit24(uint32_t x) { return (float)(x >> 8) * 5.9604644775390625e-08f; }

typedef struct { uint32_t pixelHash, index, dim; } sampler;

static void sampler_start(sampler* s, uint64_t seed, int px, int py, int index) {
    uint32_t h = mix((uint32_t)seed ^ mix((uint32_t)(seed >> 32)));
    h = hcomb(h, (uint32_t)px);
    s->pixelHash = hcomb(h, (uint32_t)py);
    s->index = (uint32_t)index;
    s->dim = 0;
}
static void get2(sampler* s, float* x, float* y) {
    const uint32_t sd = hcomb(s->pixelHash, s->dim++);
    const uint32_t index = nus(s->index, sd);
    *x = unit24(nus(rev(index), hcomb(sd, 0u)));
    *y = unit24(nus(sobol1(index), hcomb(sd, 1u)));
}
static float get1(sampler* s) {
    float x, y;
    get2(s, &x, &y); /* a 1-D request spends a dimension and equals get2D().x */
    return x;
}

int32_t po_sobol(uint64_t seed, int32_t px, int32_t py, int32_t index, int32_t ndims, float* out) {
    sampler s;
    sampler_start(&s, seed, px, py, index);
    for (int k = 0; k < ndims; ++k) get2(&s, &out[2 * k], &out[2 * k + 1]);
    return 0;
}

/* ---- scene ------------------------------------------------------------------------------- */
typedef struct {
    v3 p0, p1, p2, n0, n1, n2;
    v3 albedo, emission;
    int light;  /* light index of this triangle, -1 if not emissive */
} tri;

typedef struct {
    tri* t;
    int n, cap;
    int nLights;
    int* lightTri; /* light index -> triangle */
} scene;

void* po_scene_create(void) { return calloc(1, sizeof(scene)); }
void po_scene_destroy(void* p) {
    scene* s = (scene*)p;
    if (!s) return;
    free(s->t);
    free(s->lightTri);
    free(s);
}

/* A Lambert mesh; vertex normals computed as TriangleMesh::calculateNormals does. */
int32_t po_scene_add_mesh(void* p, const float* pos, uint32_t nv, const uint32_t* idx, uint32_t nt, const float* albedo,
                          const float* emission) {
    scene* s = (scene*)p;
    v3* nrm = (v3*)calloc(nv ? nv : 1, sizeof(v3));
    for (uint32_t i = 0; i < nt; ++i) {
        const uint32_t a = idx[3 * i], b = idx[3 * i + 1], c = idx[3 * i + 2];
        const v3 A = mk(pos[3 * a], pos[3 * a + 1], pos[3 * a + 2]);
        const v3 B = mk(pos[3 * b], pos[3 * b + 1], pos[3 * b + 2]);
        const v3 Cc = mk(pos[3 * c], pos[3 * c + 1], pos[3 * c + 2]);
        const v3 n = cross(sub(B, A), sub(Cc, A));
        nrm[a] = add(nrm[a], n);
        nrm[b] = add(nrm[b], n);
        nrm[c] = add(nrm[c], n);
    }
    for (uint32_t i = 0; i < nv; ++i)
        if (len2(nrm[i]) > 0.0f) nrm[i] = normalize(nrm[i]);
    const int emissive = emission[0] != 0.0f || emission[1] != 0.0f || emission[2] != 0.0f;
    for (uint32_t i = 0; i < nt; ++i) {
        if (s->n == s->cap) {
            s->cap = s->cap ? 2 * s->cap : 64;
            s->t = (tri*)realloc(s->t, (size_t)s->cap * sizeof(tri));
        }
        tri* T = &s->t[s->n++];
        const uint32_t a = idx[3 * i], b = idx[3 * i + 1], c = idx[3 * i + 2];
        T->p0 = mk(pos[3 * a], pos[3 * a + 1], pos[3 * a + 2]);
        T->p1 = mk(pos[3 * b], pos[3 * b + 1], pos[3 * b + 2]);
        T->p2 = mk(pos[3 * c], pos[3 * c + 1], pos[3 * c + 2]);
        T->n0 = nrm[a];
        T->n1 = nrm[b];
        T->n2 = nrm[c];
        T->albedo = mk(albedo[0], albedo[1], albedo[2]);
        T->emission = mk(emission[0], emission[1], emission[2]);
        T->light = -1;
        if (emissive) {
            s->lightTri = (int*)realloc(s->lightTri, (size_t)(s->nLights + 1) * sizeof(int));
            s->lightTri[s->nLights] = s->n - 1;
            T->light = s->nLights++;
        }
    }
    free(nrm);
    return 0;
}

/* ---- intersection ------------------------------------------------------------------------ */
/* BVH::hitTriangleLean (bvh.cpp:302-316) */
static int tri_hit(const tri* T, v3 o, v3 d, float tMin, float tMax, float* t, float* uu, float* vv) {
    const v3 e1 = sub(T->p1, T->p0), e2 = sub(T->p2, T->p0);
    const float eps = 1e-14f * len2(e1) * len2(e2);
    const v3 h = cross(d, e2);
    const float a = dot(e1, h);
    if (a * a <= eps) return 0;
    const float f = 1.0f / a;
    const v3 s = sub(o, T->p0);
    const float u = f * dot(s, h);
    if (!(u >= 0.0f && u <= 1.0f)) return 0;
    const v3 q = cross(s, e1);
    const float v = f * dot(d, q);
    if (!(v >= 0.0f && u + v <= 1.0f)) return 0;
    *t = f * dot(e2, q);
    *uu = u;
    *vv = v;
    return *t >= tMin && *t <= tMax;
}

static int closest(const scene* S, v3 o, v3 d, float* tOut, float* uOut, float* vOut) {
    int best = -1;
    float tMax = 1e30f;
    for (int i = 0; i < S->n; ++i) {
        float t, u, v;
        if (tri_hit(&S->t[i], o, d, 0.0f, tMax, &t, &u, &v)) {
            tMax = t;
            best = i;
            *tOut = t;
            *uOut = u;
            *vOut = v;
        }
    }
    return best;
}

static int any_hit(const scene* S, v3 o, v3 d, float tMax) {
    for (int i = 0; i < S->n; ++i) {
        float t, u, v;
        if (tri_hit(&S->t[i], o, d, 0.0f, tMax, &t, &u, &v)) return 1;
    }
    return 0;
}

typedef struct {
    v3 point, normal, ng, pError, pSmooth;
    int front, hasSmooth, tri;
} isect;

static float gammaN(int n) {
    const float eps = 5.9604645e-8f;
    return ((float)n * eps) / (1.0f - (float)n * eps);
}

/* Triangle::fillHit (triangle.cpp:54-100), the fields the Lambert path reads */
static void fill_hit(const tri* T, int index, v3 d, float u, float v, isect* is) {
    const v3 e1 = sub(T->p1, T->p0), e2 = sub(T->p2, T->p0);
    const float w = 1.0f - u - v;
    const v3 a0 = muls(T->p0, w), a1 = muls(T->p1, u), a2 = muls(T->p2, v);
    is->point = add(add(a0, a1), a2);
    const float iso = gammaN(32) * fmax2(fmax2(fmax2(maxc(vabs(T->p0)), maxc(vabs(T->p1))), maxc(vabs(T->p2))), 1e-20f);
    is->pError = add(muls(add(add(vabs(a0), vabs(a1)), vabs(a2)), gammaN(16)), mk(iso, iso, iso));
    const v3 g = normalize(cross(e1, e2));
    const int hasN = len2(T->n0) > 0.0f && len2(T->n1) > 0.0f && len2(T->n2) > 0.0f;
    const v3 sh = hasN ? normalize(add(add(muls(T->n0, w), muls(T->n1, u)), muls(T->n2, v))) : g;
    is->ng = g;
    is->front = dot(d, sh) < 0.0f;
    is->normal = is->front ? sh : neg(sh);
    if (len2(is->ng) == 0.0f) is->ng = sh;
    is->hasSmooth = 0;
    if (hasN) {
        const v3 p = is->point;
        const v3 m0 = normalize(T->n0), m1 = normalize(T->n1), m2 = normalize(T->n2);
        const v3 lift = add(add(muls(m0, w * fmax2(0.0f, dot(sub(T->p0, p), m0))),
                                muls(m1, u * fmax2(0.0f, dot(sub(T->p1, p), m1)))),
                            muls(m2, v * fmax2(0.0f, dot(sub(T->p2, p), m2))));
        if (len2(lift) > 0.0f) {
            is->pSmooth = add(p, lift);
            is->hasSmooth = 1;
        }
    }
    is->tri = index;
}

/* ray_spawn.h:25-87 */
static float next_up(float v) {
    uint32_t u;
    if (!finite1(v) && v > 0.0f) return v;
    if (v == -0.0f) v = 0.0f;
    memcpy(&u, &v, 4);
    if (v >= 0.0f) ++u; else --u;
    memcpy(&v, &u, 4);
    return v;
}
static float next_down(float v) {
    uint32_t u;
    if (!finite1(v) && v < 0.0f) return v;
    if (v == 0.0f) v = -0.0f;
    memcpy(&u, &v, 4);
    if (v > 0.0f) --u; else ++u;
    memcpy(&v, &u, 4);
    return v;
}
static v3 offset_origin(v3 p, v3 pErr, v3 n, v3 w) {
    const float d = dot(vabs(n), pErr);
    v3 off = muls(n, d);
    if (dot(w, n) < 0.0f) off = neg(off);
    v3 po = add(p, off);
    po.x = off.x > 0.0f ? next_up(po.x) : (off.x < 0.0f ? next_down(po.x) : po.x);
    po.y = off.y > 0.0f ? next_up(po.y) : (off.y < 0.0f ? next_down(po.y) : po.y);
    po.z = off.z > 0.0f ? next_up(po.z) : (off.z < 0.0f ? next_down(po.z) : po.z);
    return po;
}
static v3 spawn_n(const isect* is) { return len2(is->ng) > 0.0f ? is->ng : is->normal; }
static v3 shadow_origin(const isect* is, v3 L) {
    const v3 n = spawn_n(is);
    v3 p = is->point;
    if (is->hasSmooth) {
        const v3 so = is->front ? is->normal : neg(is->normal);
        const v3 go = dot(n, so) >= 0.0f ? n : neg(n);
        const float NL = dot(so, L);
        if (NL > 0.0f) {
            const float NgL = dot(go, L);
            float amount = NL < 0.1f ? 2.0f - (NgL + NL) / 0.1f : 1.0f - NgL / 0.1f;
            amount = amount < 0.0f ? 0.0f : (amount > 1.0f ? 1.0f : amount);
            if (amount > 0.0f) p = add(p, muls(sub(is->pSmooth, is->point), amount));
        }
    }
    return offset_origin(p, is->pError, n, L);
}

/* ---- lights, Lambert ---------------------------------------------------------------------- */
static float tri_area(const tri* T, v3* nOut) {
    const v3 n = cross(sub(T->p1, T->p0), sub(T->p2, T->p0));
    const float l = sqrtf(len2(n));
    *nOut = l > 0.0f ? divs(n, l) : mk(0, 1, 0);
    return 0.5f * l;
}
static float solid_pdf(float d2, float c, float area) {
    if (!(c > 1e-6f) || !(area > 0.0f) || !(d2 > 0.0f)) return 0.0f;
    return d2 / (area * c);
}
static float importance(const tri* T, v3 p, v3 n) {
    v3 ln;
    const float area = tri_area(T, &ln);
    const v3 d = sub(muls(add(add(T->p0, T->p1), T->p2), 1.0f / 3.0f), p);
    const float d2 = len2(d);
    const float L = fmax2(0.0f, lum(T->emission));
    if (!(d2 > 0.0f)) return L * (2.0f * PI);
    const v3 w = divs(d, sqrtf(d2));
    const float cl = fmax2(fabsf(dot(w, ln)), 0.2f);
    const float omega = fmin2(area * cl / d2, 2.0f * PI);
    const float rc = dot(n, w);
    return L * omega * (rc > 0.05f ? rc : 0.05f);
}

typedef struct {
    float pmf[64];
    int uniform, valid;
} picker;

static void prepare(const scene* S, v3 p, v3 n, picker* c) {
    const int count = S->nLights;
    c->valid = 1;
    c->uniform = 1;
    if (count <= 1) return;
    float sum = 0.0f;
    for (int i = 0; i < count; ++i) {
        const float w = importance(&S->t[S->lightTri[i]], p, n);
        c->pmf[i] = (w > 0.0f && finite1(w)) ? w : 0.0f;
    }
    for (int i = 0; i < count; ++i) sum += c->pmf[i];
    if (!(sum > 0.0f) || !finite1(sum)) {
        for (int i = 0; i < count; ++i) c->pmf[i] = 1.0f / (float)count;
    } else {
        const float a = (1.0f - 0.15f) / sum, b = 0.15f / (float)count;
        for (int i = 0; i < count; ++i) c->pmf[i] = c->pmf[i] * a + b;
    }
    c->uniform = 0;
}
static int pick(const scene* S, const picker* c, float u, float* pmf) {
    const int n = S->nLights;
    *pmf = 0.0f;
    if (!c->valid || n <= 0) return -1;
    if (c->uniform) {
        int k = (int)(u * (float)n);
        *pmf = 1.0f / (float)n;
        return k < n - 1 ? k : n - 1;
    }
    float acc = 0.0f;
    int k = n - 1;
    for (int i = 0; i < n - 1; ++i) {
        if (u < acc + c->pmf[i]) { k = i; break; }
        acc += c->pmf[i];
    }
    *pmf = c->pmf[k];
    return k;
}
static float pick_pmf(const scene* S, const picker* c, int index) {
    if (!c->valid || index < 0 || index >= S->nLights) return 0.0f;
    if (c->uniform) return 1.0f / (float)S->nLights;
    return c->pmf[index];
}

static void disk(float ux, float uy, float* dx, float* dy) {
    const float sx = 2.0f * ux - 1.0f, sy = 2.0f * uy - 1.0f;
    float r, th;
    if (sx == 0.0f && sy == 0.0f) { *dx = 0.0f; *dy = 0.0f; return; }
    if (fabsf(sx) > fabsf(sy)) { r = sx; th = (PI / 4.0f) * (sy / sx); }
    else { r = sy; th = (PI / 2.0f) - (PI / 4.0f) * (sx / sy); }
    *dx = r * cosf(th);
    *dy = r * sinf(th);
}
typedef struct { v3 s, t, n; } frame;
static frame make_frame(v3 n) {
    frame f;
    const float sign = copysignf(1.0f, n.z);
    const float a = -1.0f / (sign + n.z);
    const float b = n.x * n.y * a;
    f.n = n;
    f.s = mk(1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x);
    f.t = mk(b, sign + n.y * n.y * a, -n.y);
    return f;
}
static v3 to_local(frame f, v3 v) { return mk(dot(v, f.s), dot(v, f.t), dot(v, f.n)); }
static v3 to_world(frame f, v3 v) { return add(add(muls(f.s, v.x), muls(f.t, v.y)), muls(f.n, v.z)); }
static float power_h(int nf, float fp, int ng, float gp) {
    const float f = (float)nf * fp, g = (float)ng * gp, f2 = f * f;
    return f2 / (f2 + g * g);
}

/* ---- estimator ----------------------------------------------------------------------------- */
typedef struct {
    float position[3], lower_left[3], horizontal[3], vertical[3];
} camdesc;

static v3 Li(const scene* S, v3 ro, v3 rd, sampler* sm, int maxDepth, int rrDepth) {
    v3 L = mk(0, 0, 0), thr = mk(1, 1, 1);
    int specular = 1, depth = 0;
    float lastPdf = 0.0f;
    v3 lastPoint = ro;
    picker pk;
    pk.valid = 0;
    pk.uniform = 1;
    for (;;) {
        float t, u, v;
        const int h = closest(S, ro, rd, &t, &u, &v);
        if (h < 0) break; /* no environment in this scene */
        isect is;
        fill_hit(&S->t[h], h, rd, u, v, &is);
        const tri* T = &S->t[h];
        const v3 wo = neg(rd);
        if (!black(T->emission)) {
            float weight = 1.0f;
            if (!specular) {
                float lightPdf = 0.0f;
                if (T->light >= 0) {
                    v3 ln;
                    const float area = tri_area(T, &ln);
                    const v3 toL = sub(is.point, lastPoint);
                    const float d2 = len2(toL);
                    const float pdfHit = d2 > 0.0f ? solid_pdf(d2, fabsf(dot(divs(toL, sqrtf(d2)), ln)), area) : 0.0f;
                    lightPdf = pick_pmf(S, &pk, T->light) * pdfHit;
                }
                if (lightPdf > 0.0f && lastPdf > 0.0f) weight = power_h(1, lastPdf, 1, lightPdf);
            }
            const v3 c = mulv(thr, muls(T->emission, weight));
            if (finite3(c)) L = add(L, c);
        }
        if (depth >= maxDepth) break;
        /* NEE */
        if (S->nLights > 0) {
            prepare(S, is.point, is.normal, &pk);
            float pmf;
            const int li = pick(S, &pk, get1(sm), &pmf);
            float ux, uy;
            get2(sm, &ux, &uy);
            if (li >= 0 && pmf > 0.0f) {
                const tri* LT = &S->t[S->lightTri[li]];
                v3 ln;
                const float area = tri_area(LT, &ln);
                if (area > 0.0f && !black(LT->emission)) {
                    const float su0 = sqrtf(ux);
                    const float b1 = 1.0f - su0, b2 = uy * su0;
                    const v3 pL = add(add(muls(LT->p0, 1.0f - b1 - b2), muls(LT->p1, b1)), muls(LT->p2, b2));
                    const v3 toL = sub(pL, is.point);
                    const float d2 = len2(toL);
                    const float dist = sqrtf(d2);
                    if (dist > 0.0f) {
                        const v3 wi = divs(toL, dist);
                        const float lpdf = solid_pdf(d2, fabsf(dot(wi, ln)), area);
                        if (lpdf > 0.0f) {
                            /* spawnRayTo (ray_spawn.h:75-85) */
                            const v3 target = add(is.point, muls(wi, dist));
                            const v3 tt = sub(target, is.point);
                            const float tl = sqrtf(len2(tt));
                            if (tl > 0.0f) {
                                const v3 so = shadow_origin(&is, divs(tt, tl));
                                const v3 dd = sub(target, so);
                                const float sd = sqrtf(len2(dd));
                                const float slack = fmax2(sd * 1e-4f, 2e-6f * maxc(vabs(target)));
                                if (sd > slack && !any_hit(S, so, divs(dd, sd), sd - slack)) {
                                    const frame f = make_frame(is.normal);
                                    const float ci = to_local(f, wi).z, co = to_local(f, wo).z;
                                    const v3 fr = muls(T->albedo, 1.0f / PI);
                                    if (ci > 0.0f && co > 0.0f && !black(fr)) {
                                        const float bpdf = ci * (1.0f / PI);
                                        const float cosT = fabsf(dot(wi, is.normal));
                                        const float lightPdf = pmf * lpdf;
                                        const float w = power_h(1, lightPdf, 1, bpdf);
                                        const v3 nee = muls(mulv(mulv(fr, LT->emission), mk(1, 1, 1)), cosT * w / (lightPdf * 1.0f));
                                        const v3 c = mulv(thr, nee);
                                        if (finite3(c)) L = add(L, c);
                                    }
                                }
                            }
                        }
                    }
                }
            }
        }
        /* BSDF sample (Lambertian::sample) */
        (void)get1(sm);
        float u1, u2;
        get2(sm, &u1, &u2);
        const frame f = make_frame(is.normal);
        if (to_local(f, wo).z <= 0.0f) break;
        float dx, dy;
        disk(u1, u2, &dx, &dy);
        const v3 wl = mk(dx, dy, sqrtf(fmax2(0.0f, 1.0f - dx * dx - dy * dy)));
        const v3 wi = normalize(to_world(f, wl));
        if (wl.z <= 0.0f) break;
        const v3 fr = muls(T->albedo, 1.0f / PI);
        const float pdf = wl.z * (1.0f / PI);
        if (pdf <= 0.0f || black(fr)) break; /* path_tracer.cpp:767 */
        const float cosT = fabsf(dot(wi, is.normal));
        thr = mulv(thr, muls(fr, cosT / pdf));
        if (!finite3(thr)) break;
        lastPdf = pdf;
        lastPoint = is.point;
        specular = 0;
        ro = offset_origin(is.point, is.pError, spawn_n(&is), wi);
        rd = wi;
        ++depth;
        if (depth > rrDepth) {
            const float m = fmax2(fmax2(thr.x, thr.y), thr.z);
            if (!(m >= 1.0f)) {
                if (!(m > 0.0f) || get1(sm) >= m) break;
                thr = divs(thr, m);
            }
        }
    }
    return L;
}

static void camera_ray(const camdesc* c, int x, int y, int w, int h, sampler* s, v3* o, v3* d) {
    float ux, uy, lx, ly;
    get2(s, &ux, &uy);
    const float sx = ((float)x + 0.5f + (ux - 0.5f) * 1.0f) / (float)w;
    const float sy = 1.0f - ((float)y + 0.5f + (uy - 0.5f) * 1.0f) / (float)h;
    get2(s, &lx, &ly);
    const v3 pos = mk(c->position[0], c->position[1], c->position[2]);
    const v3 ll = mk(c->lower_left[0], c->lower_left[1], c->lower_left[2]);
    const v3 hz = mk(c->horizontal[0], c->horizontal[1], c->horizontal[2]);
    const v3 vt = mk(c->vertical[0], c->vertical[1], c->vertical[2]);
    const v3 target = add(add(ll, muls(hz, sx)), muls(vt, sy));
    *o = pos;
    *d = normalize(sub(target, pos));
}

/* Primary hit of pixel (x, y), sample `index`: triangle index (insertion order) or -1, and t. */
int32_t po_trace_primary(void* p, const camdesc* cam, int32_t w, int32_t h, uint64_t seed, int32_t index,
                         int32_t* outTri, float* outT) {
    const scene* S = (const scene*)p;
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            sampler s;
            sampler_start(&s, seed, x, y, index);
            v3 o, d;
            camera_ray(cam, x, y, w, h, &s, &o, &d);
            float t = 0.0f, u, v;
            const int k = closest(S, o, d, &t, &u, &v);
            outTri[y * w + x] = k;
            outT[y * w + x] = k >= 0 ? t : 0.0f;
        }
    return 0;
}

/* Mean image of samples [first, first+count): rows [y0, y1) of a w x h film (box filter width 1). */
int32_t po_render(void* p, const camdesc* cam, int32_t w, int32_t h, uint64_t seed, int32_t maxDepth, int32_t rrDepth,
                  int32_t first, int32_t count, int32_t y0, int32_t y1, float* mean) {
    const scene* S = (const scene*)p;
    for (int y = y0; y < y1; ++y)
        for (int x = 0; x < w; ++x) {
            v3 sum = mk(0, 0, 0);
            uint32_t n = 0;
            for (int si = first; si < first + count; ++si) {
                sampler s;
                sampler_start(&s, seed, x, y, si);
                v3 o, d;
                camera_ray(cam, x, y, w, h, &s, &o, &d);
                const v3 c = Li(S, o, d, &s, maxDepth, rrDepth);
                ++n;
                if (finite3(c) && c.x >= 0.0f && c.y >= 0.0f && c.z >= 0.0f) sum = add(sum, c);
            }
            const float inv = n ? 1.0f / (float)n : 0.0f;
            mean[3 * (y * w + x) + 0] = sum.x * inv;
            mean[3 * (y * w + x) + 1] = sum.y * inv;
            mean[3 * (y * w + x) + 2] = sum.z * inv;
        }
    return 0;
}
