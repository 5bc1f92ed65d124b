/*
 * Test infrastructure only: the oracle (see bh_oracle.h). Never linked into
 * the product. Every arithmetic step below follows the reference's DOUBLE
 * build in the same order so that results are bit-identical to it; each
 * function cites the reference lines it restates.
 */
#define _GNU_SOURCE
#include "bh_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define BHO_G 6.67384e-11 /* src/main.cpp:322 */

/* ---------------------------------------------------------------- generator */
/* std::default_random_engine is minstd_rand0 in libstdc++: x <- 16807 x mod
 * (2^31 - 1), seeded with s mod m (1 when that is 0). */
typedef struct { uint64_t x; } minstd;

static void minstd_seed(minstd *g, unsigned long s) {
    uint64_t m = 2147483647u;
    g->x = (uint64_t)s % m;
    if (g->x == 0) g->x = 1;
}

static uint64_t minstd_next(minstd *g) {
    g->x = (g->x * 16807u) % 2147483647u;
    return g->x;
}

/* libstdc++ generate_canonical<double, 53>: two draws (range r = 2^31 - 2,
 * floor(log2 r) = 30 bits each), sum = d0 + d1 * r, scaled by 1/r^2 where
 * r^2 is formed in long double and rounded to double. */
static double canonical(minstd *g) {
    const long double r = 2147483646.0L;
    double sum = 0.0, tmp = 1.0;
    for (int k = 0; k < 2; k++) {
        sum += (double)(minstd_next(g) - 1u) * tmp;
        tmp = (double)((long double)tmp * r);
    }
    double ret = sum / tmp;
    if (ret >= 1.0) ret = nextafter(1.0, 0.0);
    return ret;
}

static double uniform(minstd *g, double a, double b) { return canonical(g) * (b - a) + a; }

/* normal_distribution (Marsaglia polar, one cached value per distribution
 * object). The reference creates the object per random_datatype call, so the
 * cache lives for one call's rejection loop only. */
typedef struct { int saved_ok; double saved; } normal_state;

static double normal_draw(minstd *g, normal_state *st, double mean, double sd) {
    double ret;
    if (st->saved_ok) {
        st->saved_ok = 0;
        ret = st->saved;
    } else {
        double x, y, r2;
        do {
            x = 2.0 * canonical(g) - 1.0;
            y = 2.0 * canonical(g) - 1.0;
            r2 = x * x + y * y;
        } while (r2 > 1.0 || r2 == 0.0);
        double mult = sqrt(-2 * log(r2) / r2);
        st->saved = x * mult;
        st->saved_ok = 1;
        ret = y * mult;
    }
    return ret * sd + mean;
}

/* random_datatype, src/main.cpp:184-218. */
static double random_value(minstd *g, double low, double high, int dist) {
    double r = -1;
    if (dist == 0) {
        r = uniform(g, low, high);
    } else if (dist == 1) {
        double lambda = -1.0 * log(0.001) / (high - low);
        do {
            r = -log(1.0 - canonical(g)) / lambda + low;
        } while (r > high || r < low);
    } else {
        double center = (high + low) / 2.0;
        double deviation = (high - low) / 6.0;
        normal_state st = {0, 0.0};
        do {
            r = normal_draw(g, &st, center, deviation);
        } while (r > high || r < low);
    }
    return r;
}

/* random_vector, src/main.cpp:220-224. GCC evaluates the three constructor
 * arguments right to left, so the draws land in z, y, x order. */
static void random_vec(minstd *g, double low, double high, double *v) {
    v[2] = random_value(g, low, high, 0);
    v[1] = random_value(g, low, high, 0);
    v[0] = random_value(g, low, high, 0);
}

static double magnitude3(const double *v) {
    return sqrt(pow(v[0], 2) + pow(v[1], 2) + pow(v[2], 2));
}

/* generate_particle, src/main.cpp:226-275. */
int bho_generate(const bho_gen_params *p, uint32_t n, double *pos, double *vel, double *mass) {
    minstd g;
    minstd_seed(&g, p->seed);
    for (uint32_t i = 0; i < n; i++) {
        double m = random_value(&g, p->min_mass, p->max_mass, p->mass_dist);
        double x[3], v[3];
        if (p->gen_type == 0) {
            random_vec(&g, -1 * (p->size / 2), p->size / 2, x);
            x[0] *= p->scale_x; x[1] *= p->scale_y; x[2] *= p->scale_z;
            random_vec(&g, -1, 1, v);
            double mag = magnitude3(v);
            v[0] /= mag; v[1] /= mag; v[2] /= mag;
            double s = random_value(&g, p->min_vel, p->max_vel, p->vel_dist);
            v[0] *= s; v[1] *= s; v[2] *= s;
        } else if (p->gen_type == 1 || p->gen_type == 2) {
            double radius;
            if (p->gen_type == 1) {
                radius = random_value(&g, 0, 1, 0);
                radius = cbrt(radius) * p->r_sphere;
            } else {
                radius = p->r_sphere;
            }
            double th = random_value(&g, 0, 6.28318530718, 0);
            double az = acos(random_value(&g, -1, 1, 0));
            x[0] = radius * sin(az) * cos(th);
            x[1] = radius * sin(az) * sin(th);
            x[2] = radius * cos(az);
            x[0] *= p->scale_x; x[1] *= p->scale_y; x[2] *= p->scale_z;
            double rot[3] = {p->rot_x, p->rot_y, p->rot_z};
            double mag = magnitude3(rot);
            rot[0] /= mag; rot[1] /= mag; rot[2] /= mag;
            rot[0] *= p->rotation_magnitude; rot[1] *= p->rotation_magnitude;
            rot[2] *= p->rotation_magnitude;
            v[0] = rot[1] * x[2] - rot[2] * x[1];
            v[1] = rot[2] * x[0] - rot[0] * x[2];
            v[2] = rot[0] * x[1] - rot[1] * x[0];
        } else {
            return -1;
        }
        pos[3 * i] = x[0]; pos[3 * i + 1] = x[1]; pos[3 * i + 2] = x[2];
        vel[3 * i] = v[0]; vel[3 * i + 1] = v[1]; vel[3 * i + 2] = v[2];
        mass[i] = m;
    }
    return 0;
}

/* --------------------------------------------------------------------- tree */
typedef struct {
    double center[3], com[3], side, mass;
    int32_t child[8];
    int32_t p; /* particle index or -1 */
} bho_node;

struct bho_tree {
    uint32_t n;
    const double *pos;
    const double *mass;
    bho_node *nodes;
    int64_t count, cap;
    int depth;
    int single; /* the reference's FLOAT build: every value below is a float */
};

/* In a FLOAT tree positions and masses enter as floats, as the reference
 * harness converts them (datatype). */
static double in_pos(const bho_tree *t, size_t i, int k) {
    const double v = t->pos[3 * i + k];
    return t->single ? (double)(float)v : v;
}
static double in_mass(const bho_tree *t, size_t i) {
    const double v = t->mass[i];
    return t->single ? (double)(float)v : v;
}

/* Root cube, src/main.cpp:889-920: bbox midpoint; side = largest extent + 2,
 * a tie for the largest extent falls through to the z extent. */
void bho_root_cube(uint32_t n, const double *pos, double *center, double *side) {
    double mn[3] = {1.7976931348623157e308, 1.7976931348623157e308, 1.7976931348623157e308};
    double mx[3] = {-1.7976931348623157e308, -1.7976931348623157e308, -1.7976931348623157e308};
    for (uint32_t i = 0; i < n; i++)
        for (int k = 0; k < 3; k++) {
            double v = pos[3 * i + k];
            if (v < mn[k]) mn[k] = v;
            if (v > mx[k]) mx[k] = v;
        }
    for (int k = 0; k < 3; k++) center[k] = (mn[k] + mx[k]) / 2.0;
    double ex = mx[0] - mn[0], ey = mx[1] - mn[1], ez = mx[2] - mn[2];
    if (ex > ey && ex > ez) *side = ex + 2.0;
    else if (ey > ex && ey > ez) *side = ey + 2.0;
    else *side = ez + 2.0;
}

/* The same in the FLOAT build (src/main.cpp:889-920 with datatype float): float
 * extrema; center = float(min + max) / 2.0 (exact halving, back to float);
 * side = float(float(max - min) + 2.0); the extent comparisons in float. */
void bho_root_cube_f32(uint32_t n, const double *pos, double *center, double *side) {
    float mn[3] = {3.40282347e38f, 3.40282347e38f, 3.40282347e38f};
    float mx[3] = {-3.40282347e38f, -3.40282347e38f, -3.40282347e38f};
    for (uint32_t i = 0; i < n; i++)
        for (int k = 0; k < 3; k++) {
            float v = (float)pos[3 * i + k];
            if (v < mn[k]) mn[k] = v;
            if (v > mx[k]) mx[k] = v;
        }
    for (int k = 0; k < 3; k++) center[k] = (double)(float)((double)(mn[k] + mx[k]) / 2.0);
    float ex = mx[0] - mn[0], ey = mx[1] - mn[1], ez = mx[2] - mn[2];
    float s;
    if (ex > ey && ex > ez) s = (float)((double)ex + 2.0);
    else if (ey > ex && ey > ez) s = (float)((double)ey + 2.0);
    else s = (float)((double)ez + 2.0);
    *side = (double)s;
}

static int32_t new_node(bho_tree *t, const double *center, double side) {
    if (t->count == t->cap) {
        int64_t nc = t->cap ? 2 * t->cap : 1024;
        bho_node *nn = (bho_node *)realloc(t->nodes, (size_t)nc * sizeof(bho_node));
        if (!nn) return -1;
        t->nodes = nn;
        t->cap = nc;
    }
    bho_node *d = &t->nodes[t->count];
    for (int k = 0; k < 3; k++) { d->center[k] = center[k]; d->com[k] = center[k]; }
    d->side = side;
    d->mass = 0;
    for (int k = 0; k < 8; k++) d->child[k] = -1;
    d->p = -1;
    return (int32_t)t->count++;
}

/* Octant: x bit 1, y bit 2, z bit 4, strict '>' (src/octree.cpp:153-165). */
static int octant(const bho_tree *t, int32_t par, const double *c) {
    int i = 0;
    if (in_pos(t, (size_t)par, 0) > c[0]) i += 1;
    if (in_pos(t, (size_t)par, 1) > c[1]) i += 2;
    if (in_pos(t, (size_t)par, 2) > c[2]) i += 4;
    return i;
}

/* allocate_child, src/octree.cpp:54-85: center += (+-half/2) per axis. */
static int32_t alloc_child(bho_tree *t, int32_t node, int i) {
    int sx = (i & 1) ? 1 : -1, sy = (i & 2) ? 1 : -1, sz = (i & 4) ? 1 : -1;
    double c[3], half;
    if (t->single) {
        float h = (float)t->nodes[node].side / 2;
        c[0] = (float)t->nodes[node].center[0] + sx * h / 2;
        c[1] = (float)t->nodes[node].center[1] + sy * h / 2;
        c[2] = (float)t->nodes[node].center[2] + sz * h / 2;
        half = h;
    } else {
        half = t->nodes[node].side / 2;
        c[0] = t->nodes[node].center[0] + sx * half / 2;
        c[1] = t->nodes[node].center[1] + sy * half / 2;
        c[2] = t->nodes[node].center[2] + sz * half / 2;
    }
    int32_t k = new_node(t, c, half);
    if (k >= 0) t->nodes[node].child[i] = k;
    return k;
}

#define BHO_MAX_DEPTH 2000

/* add_particle, src/octree.cpp:134-196 (iterative form of the same recursion). */
static int add_particle(bho_tree *t, int32_t node, int32_t par, int level) {
    for (;;) {
        if (level > BHO_MAX_DEPTH) return -2; /* coincident particles */
        if (level > t->depth) t->depth = level;
        bho_node *d = &t->nodes[node];
        if (d->p < 0) {
            int leaf = 1;
            for (int k = 0; k < 8; k++)
                if (d->child[k] >= 0) { leaf = 0; break; }
            if (leaf) { d->p = par; return 0; }
            int i = octant(t, par, d->center);
            if (d->child[i] < 0 && alloc_child(t, node, i) < 0) return -1;
            node = t->nodes[node].child[i];
            level++;
        } else {
            int32_t q = d->p;
            int i = octant(t, q, d->center);
            int32_t c = t->nodes[node].child[i];
            if (c < 0 && (c = alloc_child(t, node, i)) < 0) return -1;
            if (level + 1 > t->depth) t->depth = level + 1;
            t->nodes[c].p = q; /* the fresh child is an empty leaf */
            t->nodes[node].p = -1;
        }
    }
}

/* calc_mass + calc_com, src/octree.cpp:203-221 and 252-278, post-order. */
static void mass_com(bho_tree *t, int32_t node) {
    bho_node *d = &t->nodes[node];
    if (d->p >= 0) {
        d->mass = in_mass(t, (size_t)d->p);
        for (int k = 0; k < 3; k++) d->com[k] = in_pos(t, (size_t)d->p, k);
        return;
    }
    for (int i = 0; i < 8; i++) {
        int32_t c = t->nodes[node].child[i];
        if (c >= 0) mass_com(t, c);
    }
    d = &t->nodes[node];
    if (t->single) {
        /* FLOAT build: float sums in child order, float products and quotient */
        float m = 0;
        for (int i = 0; i < 8; i++)
            if (d->child[i] >= 0) m += (float)t->nodes[d->child[i]].mass;
        d->mass = m;
        if (m == 0) { d->com[0] = d->com[1] = d->com[2] = 0; return; }
        float s[3] = {0, 0, 0};
        for (int i = 0; i < 8; i++) {
            int32_t c = d->child[i];
            if (c < 0) continue;
            float cm = (float)t->nodes[c].mass;
            for (int k = 0; k < 3; k++) {
                float w = (float)t->nodes[c].com[k] * cm;
                s[k] += w;
            }
        }
        for (int k = 0; k < 3; k++) d->com[k] = s[k] / m;
        return;
    }
    double m = 0;
    for (int i = 0; i < 8; i++)
        if (d->child[i] >= 0) m += t->nodes[d->child[i]].mass;
    d->mass = m;
    if (m == 0) { d->com[0] = d->com[1] = d->com[2] = 0; return; }
    double s[3] = {0, 0, 0};
    for (int i = 0; i < 8; i++) {
        int32_t c = d->child[i];
        if (c < 0) continue;
        double cm = t->nodes[c].mass;
        s[0] += t->nodes[c].com[0] * cm;
        s[1] += t->nodes[c].com[1] * cm;
        s[2] += t->nodes[c].com[2] * cm;
    }
    d->com[0] = s[0] / m; d->com[1] = s[1] / m; d->com[2] = s[2] / m;
}

static bho_tree *build(uint32_t n, const double *pos, const double *mass, int single) {
    bho_tree *t = (bho_tree *)calloc(1, sizeof(bho_tree));
    if (!t) return NULL;
    t->n = n; t->pos = pos; t->mass = mass; t->single = single;
    double c[3], side;
    if (single) bho_root_cube_f32(n, pos, c, &side);
    else bho_root_cube(n, pos, c, &side);
    if (new_node(t, c, side) < 0) { bho_free(t); return NULL; }
    for (uint32_t i = 0; i < n; i++)
        if (add_particle(t, 0, (int32_t)i, 0) != 0) { bho_free(t); return NULL; }
    if (n > 0) mass_com(t, 0);
    return t;
}

bho_tree *bho_build_f32(uint32_t n, const double *pos, const double *mass) { return build(n, pos, mass, 1); }

bho_tree *bho_build(uint32_t n, const double *pos, const double *mass) { return build(n, pos, mass, 0); }

void bho_free(bho_tree *t) {
    if (!t) return;
    free(t->nodes);
    free(t);
}

int64_t bho_node_count(const bho_tree *t) { return t->count; }
int bho_depth(const bho_tree *t) { return t->depth; }

/* --------------------------------------------------------------------- walk */
/* distance(), src/vector.cpp:99-102, argument order (com, pos). */
static double distance3(const double *a, const double *b) {
    return sqrt(pow(a[0] - b[0], 2) + pow(a[1] - b[1], 2) + pow(a[2] - b[2], 2));
}

/* gravity(), src/main.cpp:306-333. */
static void gravity(const double *com, double nmass, const double *x, int damping, double *out) {
    double a[3] = {com[0] - x[0], com[1] - x[1], com[2] - x[2]};
    double r_sq;
    if (!damping) r_sq = pow(magnitude3(a), -2);
    else r_sq = 1.0 / (pow(magnitude3(a), 2) + exp(-1 * magnitude3(a)));
    double mag = magnitude3(a);
    a[0] /= mag; a[1] /= mag; a[2] /= mag;
    a[0] *= nmass; a[1] *= nmass; a[2] *= nmass;
    a[0] *= BHO_G; a[1] *= BHO_G; a[2] *= BHO_G;
    a[0] *= r_sq; a[1] *= r_sq; a[2] *= r_sq;
    out[0] = a[0]; out[1] = a[1]; out[2] = a[2];
}

/* The FLOAT build's distance() and gravity() (src/vector.cpp:99-109,
 * src/main.cpp:306-333 with datatype float): float differences; pow(float, 2)
 * promotes to double, so the squares and their sum are double, and sqrt's
 * double result is rounded back to float; pow(magnitude, -2) is taken in
 * double and rounded to float; exp() of a float is expf; G is rounded to float
 * by operator*=(const datatype &). */
static float magnitude_f32(float x, float y, float z) {
    return (float)sqrt(pow((double)x, 2) + pow((double)y, 2) + pow((double)z, 2));
}

static float distance_f32(const double *a, const double *b) {
    float dx = (float)a[0] - (float)b[0], dy = (float)a[1] - (float)b[1], dz = (float)a[2] - (float)b[2];
    return magnitude_f32(dx, dy, dz);
}

static void gravity_f32(const double *com, double nmass, const double *x, int damping, float *out) {
    float a[3] = {(float)com[0] - (float)x[0], (float)com[1] - (float)x[1], (float)com[2] - (float)x[2]};
    float r_sq;
    if (!damping) {
        r_sq = (float)pow((double)magnitude_f32(a[0], a[1], a[2]), -2);
    } else {
        float mg = magnitude_f32(a[0], a[1], a[2]);
        r_sq = (float)(1.0 / (pow((double)mg, 2) + (double)expf(-1 * mg)));
    }
    float mag = magnitude_f32(a[0], a[1], a[2]);
    const float m = (float)nmass, g = (float)BHO_G;
    for (int k = 0; k < 3; k++) {
        a[k] /= mag;
        a[k] *= m;
        a[k] *= g;
        a[k] *= r_sq;
        out[k] = a[k];
    }
}

typedef struct {
    const bho_tree *t;
    double theta;
    int damping;
    const uint32_t *sample;
    uint32_t m;
    uint32_t begin, end;
    double *acc;
    uint32_t *count;
    int err;
} walk_job;

/* barnes_hut_thread, src/main.cpp:368-400: BFS from the root; open iff
 * side / distance(com, pos) > theta and the node holds no particle; else add
 * gravity unless the node is the particle's own leaf. */
static void *walk_range(void *arg) {
    walk_job *j = (walk_job *)arg;
    const bho_tree *t = j->t;
    int32_t *queue = (int32_t *)malloc((size_t)(t->count + 1) * sizeof(int32_t));
    if (!queue) { j->err = -1; return NULL; }
    for (uint32_t s = j->begin; s < j->end; s++) {
        uint32_t i = j->sample ? j->sample[s] : s;
        const double x[3] = {in_pos(t, i, 0), in_pos(t, i, 1), in_pos(t, i, 2)};
        double acc[3] = {0, 0, 0};
        uint32_t cnt = 0;
        int64_t head = 0, tail = 0;
        queue[tail++] = 0;
        float facc[3] = {0, 0, 0};
        const float ftheta = (float)j->theta;
        while (head < tail) {
            const bho_node *d = &t->nodes[queue[head++]];
            int open;
            if (t->single) open = (float)d->side / distance_f32(d->com, x) > ftheta && d->p < 0;
            else open = d->side / distance3(d->com, x) > j->theta && d->p < 0;
            if (open) {
                for (int k = 0; k < 8; k++)
                    if (d->child[k] >= 0) queue[tail++] = d->child[k];
            } else if (d->p != (int32_t)i) {
                if (t->single) {
                    float g[3];
                    gravity_f32(d->com, d->mass, x, j->damping, g);
                    facc[0] += g[0]; facc[1] += g[1]; facc[2] += g[2];
                } else {
                    double g[3];
                    gravity(d->com, d->mass, x, j->damping, g);
                    acc[0] += g[0]; acc[1] += g[1]; acc[2] += g[2];
                }
                cnt++;
            }
        }
        if (t->single) { acc[0] = facc[0]; acc[1] = facc[1]; acc[2] = facc[2]; }
        j->acc[3 * (size_t)s] = acc[0];
        j->acc[3 * (size_t)s + 1] = acc[1];
        j->acc[3 * (size_t)s + 2] = acc[2];
        if (j->count) j->count[s] = cnt;
    }
    free(queue);
    return NULL;
}

int bho_forces(const bho_tree *t, double theta, int damping, int threads,
               const uint32_t *sample, uint32_t m, double *acc_out, uint32_t *count_out) {
    uint32_t total = sample ? m : t->n;
    if (total == 0) return 0;
    if (threads < 1) threads = 1;
    if ((uint32_t)threads > total) threads = (int)total;
    walk_job *jobs = (walk_job *)calloc((size_t)threads, sizeof(walk_job));
    pthread_t *th = (pthread_t *)calloc((size_t)threads, sizeof(pthread_t));
    if (!jobs || !th) { free(jobs); free(th); return -1; }
    for (int k = 0; k < threads; k++) {
        jobs[k].t = t; jobs[k].theta = theta; jobs[k].damping = damping;
        jobs[k].sample = sample; jobs[k].m = m;
        jobs[k].begin = (uint32_t)((uint64_t)total * k / threads);
        jobs[k].end = (uint32_t)((uint64_t)total * (k + 1) / threads);
        jobs[k].acc = acc_out; jobs[k].count = count_out;
        if (k > 0) pthread_create(&th[k], NULL, walk_range, &jobs[k]);
    }
    walk_range(&jobs[0]);
    int err = jobs[0].err;
    for (int k = 1; k < threads; k++) {
        pthread_join(th[k], NULL);
        if (jobs[k].err) err = jobs[k].err;
    }
    free(jobs);
    free(th);
    return err;
}

/* particle::update(dt), src/particle.cpp:66-74. */
void bho_update(uint32_t n, double *pos, double *vel, const double *acc, double dt) {
    for (size_t i = 0; i < (size_t)n; i++)
        for (int k = 0; k < 3; k++) {
            vel[3 * i + k] += acc[3 * i + k] * dt;
            pos[3 * i + k] += vel[3 * i + k] * dt;
        }
}

/* The same in the FLOAT build: temp = a * dt; v += temp; temp = v * dt; x += temp, in float. */
void bho_update_f32(uint32_t n, double *pos, double *vel, const double *acc, double dt) {
    const float fdt = (float)dt;
    for (size_t i = 0; i < (size_t)n; i++)
        for (int k = 0; k < 3; k++) {
            float v = (float)vel[3 * i + k] + (float)acc[3 * i + k] * fdt;
            float x = (float)pos[3 * i + k] + v * fdt;
            vel[3 * i + k] = v;
            pos[3 * i + k] = x;
        }
}

static int run_frames(uint32_t n, double *pos, double *vel, const double *mass, double theta, int damping,
                      double dt, int threads, uint32_t frames, double *frames_out, int single) {
    double *acc = (double *)malloc((size_t)n * 3 * sizeof(double) + 8);
    if (!acc) return -1;
    for (uint32_t f = 0; f < frames; f++) {
        bho_tree *t = build(n, pos, mass, single);
        if (!t) { free(acc); return -2; }
        int rc = bho_forces(t, theta, damping, threads, NULL, 0, acc, NULL);
        bho_free(t);
        if (rc) { free(acc); return rc; }
        if (single) bho_update_f32(n, pos, vel, acc, dt);
        else bho_update(n, pos, vel, acc, dt);
        if (frames_out) memcpy(frames_out + (size_t)f * n * 3, pos, (size_t)n * 3 * sizeof(double));
    }
    free(acc);
    return 0;
}

int bho_run_frames(uint32_t n, double *pos, double *vel, const double *mass, double theta,
                   int damping, double dt, int threads, uint32_t frames, double *frames_out) {
    return run_frames(n, pos, vel, mass, theta, damping, dt, threads, frames, frames_out, 0);
}

int bho_run_frames_f32(uint32_t n, double *pos, double *vel, const double *mass, double theta,
                       int damping, double dt, int threads, uint32_t frames, double *frames_out) {
    return run_frames(n, pos, vel, mass, theta, damping, dt, threads, frames, frames_out, 1);
}

/* ------------------------------------------------------------- direct sum */
typedef struct {
    uint32_t n;
    const double *pos, *mass;
    int damping;
    const uint32_t *targets;
    uint32_t begin, end;
    double *acc;
} direct_job;

/* Neumaier-compensated sum of the same pair formula over every other source. */
static void *direct_range(void *arg) {
    direct_job *j = (direct_job *)arg;
    for (uint32_t s = j->begin; s < j->end; s++) {
        uint32_t i = j->targets ? j->targets[s] : s;
        const double *x = &j->pos[3 * (size_t)i];
        double sum[3] = {0, 0, 0}, c[3] = {0, 0, 0};
        for (uint32_t k = 0; k < j->n; k++) {
            if (k == i) continue;
            double g[3];
            gravity(&j->pos[3 * (size_t)k], j->mass[k], x, j->damping, g);
            for (int d = 0; d < 3; d++) {
                double t = sum[d] + g[d];
                if (fabs(sum[d]) >= fabs(g[d])) c[d] += (sum[d] - t) + g[d];
                else c[d] += (g[d] - t) + sum[d];
                sum[d] = t;
            }
        }
        for (int d = 0; d < 3; d++) j->acc[3 * (size_t)s + d] = sum[d] + c[d];
    }
    return NULL;
}

int bho_direct(uint32_t n, const double *pos, const double *mass, int damping,
               const uint32_t *targets, uint32_t m, int threads, double *acc_out) {
    uint32_t total = targets ? m : n;
    if (total == 0) return 0;
    if (threads < 1) threads = 1;
    if ((uint32_t)threads > total) threads = (int)total;
    direct_job *jobs = (direct_job *)calloc((size_t)threads, sizeof(direct_job));
    pthread_t *th = (pthread_t *)calloc((size_t)threads, sizeof(pthread_t));
    if (!jobs || !th) { free(jobs); free(th); return -1; }
    for (int k = 0; k < threads; k++) {
        jobs[k].n = n; jobs[k].pos = pos; jobs[k].mass = mass; jobs[k].damping = damping;
        jobs[k].targets = targets;
        jobs[k].begin = (uint32_t)((uint64_t)total * k / threads);
        jobs[k].end = (uint32_t)((uint64_t)total * (k + 1) / threads);
        jobs[k].acc = acc_out;
        if (k > 0) pthread_create(&th[k], NULL, direct_range, &jobs[k]);
    }
    direct_range(&jobs[0]);
    for (int k = 1; k < threads; k++) pthread_join(th[k], NULL);
    free(jobs);
    free(th);
    return 0;
}

/* ------------------------------------------------------------ tree records */
typedef struct {
    const bho_tree *t;
    int cap, used;
    int *level, *count, *min_index;
    double *mass, *com, *side;
} rec_ctx;

static int rec_walk(rec_ctx *r, int32_t node, int level, int *mn_out) {
    const bho_node *d = &r->t->nodes[node];
    if (d->p >= 0) { *mn_out = d->p; return 1; }
    int slot = r->used++;
    int cnt = 0, nchild = 0, mn = 0x7fffffff;
    for (int i = 0; i < 8; i++) {
        int32_t c = d->child[i];
        if (c < 0) continue;
        int cm = 0x7fffffff;
        int cc = rec_walk(r, c, level + 1, &cm);
        if (cc > 0) nchild++;
        cnt += cc;
        if (cm < mn) mn = cm;
    }
    if (slot < r->cap) {
        r->level[slot] = (nchild >= 2 || level == 0) ? level : -1;
        r->count[slot] = cnt;
        r->min_index[slot] = mn;
        r->mass[slot] = d->mass;
        r->side[slot] = d->side;
        for (int k = 0; k < 3; k++) r->com[3 * slot + k] = d->com[k];
    }
    *mn_out = mn;
    return cnt;
}

int bho_tree_nodes(const bho_tree *t, int cap, int *level, int *count, int *min_index,
                   double *node_mass, double *com, double *side) {
    if (t->n == 0) return 0;
    rec_ctx r = {t, cap, 0, level, count, min_index, node_mass, com, side};
    int mn;
    rec_walk(&r, 0, 0, &mn);
    if (r.used > cap) return r.used;
    int kept = 0;
    for (int i = 0; i < r.used; i++) {
        if (level[i] < 0) continue;
        level[kept] = level[i]; count[kept] = count[i]; min_index[kept] = min_index[i];
        node_mass[kept] = node_mass[i]; side[kept] = side[i];
        for (int k = 0; k < 3; k++) com[3 * kept + k] = com[3 * i + k];
        kept++;
    }
    return kept;
}
