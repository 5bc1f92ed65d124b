// Drop-in replacement for fosted3/nbodysim's src/cuda_helper.cpp (and the
// src/cuda_code.cu it drives): the same C++ entry point,
//     void barnes_hut_cuda(std::unordered_set<particle*>*, octree*, bool, datatype);
//                                                      (src/cuda_helper.h:8)
// backed by the nbody_b200 library. The reference walks the tree on the host
// with 8 threads and ships 64-entry interaction chunks to the GPU per call
// (src/cuda_helper.cpp:46-246); here the particles are gathered once, the
// library builds the same octree (same root cube, same leaf rule) and runs the
// walk and the gravity sums on the GPU, and every particle's acceleration is
// overwritten with the result, as the reference's set_acc_zero +
// set_acc_offset do (src/cuda_helper.cpp:96, 190-194).
//
// Contract kept: positions, velocities and masses are read, never written;
// the `root` argument is not read (the GPU rebuilds the identical tree); a
// failure prints a message and exits with the status code, as the reference's
// handle_error does (src/cuda_code.cu:29-37).
//
// Build: compile this file with the reference's headers on the include path
// and the same -DFLOAT / -DDOUBLE as the rest of the program, and link
// libnbody_b200.so. In a FLOAT build the positions and masses are widened to
// double for the library (exactly), the library is told the program's
// datatype (nbody_params.datatype_bytes = sizeof(datatype)) so that it builds
// the tree and takes every opening decision in float as this build does, and
// the accelerations are narrowed back to float.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "cuda_helper.h"
#include "nbody_b200.h"

namespace {

struct Engine {
    nbody_ctx *ctx = nullptr;
    std::vector<particle *> order;
    std::vector<double> pos, mass, acc;
    ~Engine() {
        if (ctx) nbody_destroy(ctx);
    }
};

Engine &engine() {
    static Engine e;
    if (!e.ctx) {
        nbody_params p;
        nbody_default_params(&p);
        const char *prec = std::getenv("NBODY_B200_PRECISION");
        if (prec && prec[0] == 'f') p.precision = NBODY_PRECISION_FP64;
        p.datatype_bytes = (int)sizeof(datatype);
        int rc = nbody_create(&p, &e.ctx);
        if (rc != NBODY_OK) {
            std::fprintf(stderr, "nbody_b200: %s: %s\n", nbody_status_string(rc), nbody_last_error_message());
            std::exit(rc);
        }
    }
    return e;
}

}  // namespace

void barnes_hut_cuda(std::unordered_set<particle *> *particles, octree *root, bool damping, datatype theta) {
    (void)root;
    Engine &e = engine();
    const size_t n = particles->size();
    e.order.assign(particles->begin(), particles->end());
    e.pos.resize(3 * n);
    e.mass.resize(n);
    e.acc.resize(3 * n);
    for (size_t i = 0; i < n; i++) {
        particle *p = e.order[i];
        e.pos[3 * i] = p->get_pos()->get_x();
        e.pos[3 * i + 1] = p->get_pos()->get_y();
        e.pos[3 * i + 2] = p->get_pos()->get_z();
        e.mass[i] = p->get_mass();
    }
    int rc = nbody_barnes_hut(e.ctx, (uint32_t)n, e.pos.data(), e.mass.data(), damping ? 1 : 0, (double)theta,
                              e.acc.data(), nullptr);
    if (rc != NBODY_OK) {
        std::fprintf(stderr, "nbody_b200: %s: %s\n", nbody_status_string(rc), nbody_last_error_message());
        std::exit(rc);
    }
    for (size_t i = 0; i < n; i++) {
        particle *p = e.order[i];
        p->set_acc_zero();
        vector a((datatype)e.acc[3 * i], (datatype)e.acc[3 * i + 1], (datatype)e.acc[3 * i + 2]);
        p->set_acc_offset(&a);
    }
}
