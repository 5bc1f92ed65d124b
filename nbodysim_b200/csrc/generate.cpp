// Seeded initial conditions (host C++), the reference's generate_particle
// (src/main.cpp:184-275) with the same engine, distributions and draw order,
// so one seed yields the reference's particles bit for bit in its DOUBLE build.
// The engine and distributions are the standard library's own types, which is
// what makes the values identical; the draw order is written out explicitly:
// the reference builds its vectors with three draws as constructor arguments,
// which its GCC build evaluates right to left (z, then y, then x).
#include <cmath>
#include <random>

#include "../../include/nbody_b200.h"

namespace {

using engine = std::default_random_engine;

double draw(double low, double high, int dist, engine &g) {  // random_datatype, src/main.cpp:184-218
    double r = -1;
    if (dist == 0) {
        std::uniform_real_distribution<double> d(low, high);
        r = d(g);
    } else if (dist == 1) {
        double lambda = -1.0 * std::log(0.001) / (high - low);
        std::exponential_distribution<double> d(lambda);
        do { r = d(g) + low; } while (r > high || r < low);
    } else {
        double center = (high + low) / 2.0;
        double deviation = (high - low) / 6.0;
        std::normal_distribution<double> d(center, deviation);
        do { r = d(g); } while (r > high || r < low);
    }
    return r;
}

void draw3(double low, double high, engine &g, double *v) {  // random_vector, src/main.cpp:220-224
    v[2] = draw(low, high, 0, g);
    v[1] = draw(low, high, 0, g);
    v[0] = draw(low, high, 0, g);
}

double norm3(const double *v) { return std::sqrt(std::pow(v[0], 2) + std::pow(v[1], 2) + std::pow(v[2], 2)); }

}  // namespace

extern "C" void nbody_default_gen_params(nbody_gen_params *g) {
    // set_default, src/main.cpp:1324-1342
    g->gen_type = 0;
    g->mass_dist = 0;
    g->vel_dist = 0;
    g->size = 512;
    g->min_mass = 5e10;
    g->max_mass = 5e11;
    g->min_vel = 0;
    g->max_vel = 0;
    g->r_sphere = 100;
    g->rotation_magnitude = 0.1;
    g->rotation_vector[0] = 0; g->rotation_vector[1] = 0; g->rotation_vector[2] = 1;
    g->scale[0] = g->scale[1] = g->scale[2] = 1;
    g->seed = 0xDEADBEEFu;
}

extern "C" int nbody_generate(const nbody_gen_params *p, uint32_t n, double *pos, double *vel, double *mass) {
    if (!p || (n && (!pos || !vel || !mass))) return NBODY_ERR_INVALID;
    if (p->gen_type < 0 || p->gen_type > 2 || p->mass_dist < 0 || p->mass_dist > 2 || p->vel_dist < 0 ||
        p->vel_dist > 2)
        return NBODY_ERR_INVALID;
    if (p->scale[0] < 0 || p->scale[1] < 0 || p->scale[2] < 0) return NBODY_ERR_INVALID;
    engine g;
    g.seed((unsigned long)p->seed);
    for (uint32_t i = 0; i < n; i++) {
        double m = draw(p->min_mass, p->max_mass, p->mass_dist, g);
        double x[3], v[3];
        if (p->gen_type == 0) {
            draw3(-1 * (p->size / 2), p->size / 2, g, x);
            for (int k = 0; k < 3; k++) x[k] *= p->scale[k];
            draw3(-1, 1, g, v);
            double mag = norm3(v);
            for (int k = 0; k < 3; k++) v[k] /= mag;
            double s = draw(p->min_vel, p->max_vel, p->vel_dist, g);
            for (int k = 0; k < 3; k++) v[k] *= s;
        } else {
            double radius;
            if (p->gen_type == 1) {
                radius = draw(0, 1, 0, g);
                radius = std::cbrt(radius) * p->r_sphere;
            } else {
                radius = p->r_sphere;
            }
            double th = draw(0, 6.28318530718, 0, g);
            double az = std::acos(draw(-1, 1, 0, g));
            x[0] = radius * std::sin(az) * std::cos(th);
            x[1] = radius * std::sin(az) * std::sin(th);
            x[2] = radius * std::cos(az);
            for (int k = 0; k < 3; k++) x[k] *= p->scale[k];
            double rot[3] = {p->rotation_vector[0], p->rotation_vector[1], p->rotation_vector[2]};
            double mag = norm3(rot);
            for (int k = 0; k < 3; k++) rot[k] /= mag;
            for (int k = 0; k < 3; k++) rot[k] *= p->rotation_magnitude;
            v[0] = rot[1] * x[2] - rot[2] * x[1];  // cross(rotation, point), src/vector.cpp:117-120
            v[1] = rot[2] * x[0] - rot[0] * x[2];
            v[2] = rot[0] * x[1] - rot[1] * x[0];
        }
        for (int k = 0; k < 3; k++) {
            pos[3 * (size_t)i + k] = x[k];
            vel[3 * (size_t)i + k] = v[k];
        }
        mass[i] = m;
    }
    return NBODY_OK;
}
