/*
 * Test infrastructure only: NOT part of the product and never linked into it.
 *
 * Compiles the reference's own src/main.cpp (fosted3/nbodysim) as a library
 * so that tests and the CPU-baseline leg of bench.py can call the reference's
 * unmodified CPU path on seeded inputs:
 *   generate_particle   src/main.cpp:226-275   (seeded initial conditions)
 *   gen_root[_threaded] src/main.cpp:837-927   (root cube + octree insertion)
 *   octree::calc_mass / calc_com [_threaded]   src/octree.cpp:203-313
 *   barnes_hut_threaded src/main.cpp:432-519   (per-particle BFS walk + gravity)
 *   update_all[_threaded] src/main.cpp:929-973 (semi-implicit Euler)
 * The reference sources are compiled where they lie (see oracle/Makefile);
 * nothing from them is copied here. Its `main` is renamed so this file can
 * provide plain C entry points taking flat arrays.
 */
#define main nbodysim_reference_main
#include "main.cpp"
#undef main

#include <chrono>
#include <vector>

namespace {

struct gen_params {
    int gen_type;   /* 0 cube, 1 sphere, 2 shell (src/main.cpp:1-3) */
    int mass_dist;  /* 0 linear, 1 exp, 2 normal (src/main.cpp:4-6) */
    int vel_dist;
    double size, min_mass, max_mass, min_vel, max_vel, r_sphere, rotation_magnitude;
    double rot_x, rot_y, rot_z, scale_x, scale_y, scale_z;
    unsigned long seed;
};

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

/* Builds particles in input order; the unordered_set holds the same pointers. */
void make_particles(unsigned int n, const double *pos, const double *vel, const double *mass,
                    std::vector<particle *> &order, particle_set &set) {
    order.resize(n);
    set.reserve(n);
    for (unsigned int i = 0; i < n; i++) {
        vector p((datatype)pos[3 * i], (datatype)pos[3 * i + 1], (datatype)pos[3 * i + 2]);
        vector v(0, 0, 0);
        if (vel) v = vector((datatype)vel[3 * i], (datatype)vel[3 * i + 1], (datatype)vel[3 * i + 2]);
        vector a(0, 0, 0);
        order[i] = new particle(&p, &v, &a, (datatype)mass[i]);
        set.insert(order[i]);
    }
}

void free_particles(std::vector<particle *> &order) {
    for (particle *p : order) delete p;
    order.clear();
}

void settings_for_walk(settings &cfg, double theta, int damping, unsigned int threads) {
    set_default(cfg);
    cfg.theta = (datatype)theta;
    cfg.damping = damping != 0;
    cfg.threads = threads ? threads : 1;
    cfg.display_progress = false;
    cfg.dump_binary = cfg.dump_text = cfg.dump_image = false;
}

/* One frame's tree, exactly as main() builds it (src/main.cpp:1423-1438). */
octree *build_tree(particle_set *set, unsigned int threads, double *t_build, double *t_mass) {
    double t0 = now_s();
    octree *root = threads > 1 ? gen_root_threaded(set) : gen_root(set);
    double t1 = now_s();
    if (threads > 1) { root->calc_mass_threaded(); root->calc_com_threaded(); }
    else { root->calc_mass(); root->calc_com(); }
    double t2 = now_s();
    if (t_build) *t_build = t1 - t0;
    if (t_mass) *t_mass = t2 - t1;
    return root;
}

void delete_tree(octree *root, unsigned int threads) {
    if (threads > 1) delete_root_threaded(root);
    else delete root;
}

/* Pre-order walk recording every node that has two or more children, or the root. */
struct node_rec { int level; int count; int min_index; double mass, cx, cy, cz, side; };

int collect(octree *node, int level, const std::unordered_map<particle *, int> &index,
            std::vector<node_rec> &out, int *min_index, int *max_level) {
    if (level > *max_level) *max_level = level;
    if (node->get_particle() != NULL) {
        *min_index = index.at(node->get_particle());
        return 1;
    }
    int nchild = 0, count = 0, mn = 0x7fffffff;
    size_t slot = out.size();
    out.push_back(node_rec());
    for (unsigned int i = 0; i < 8; i++) {
        octree *c = node->get_child(i);
        if (!c) continue;
        int cmin = 0x7fffffff;
        int cc = collect(c, level + 1, index, out, &cmin, max_level);
        if (cc > 0) nchild++;
        count += cc;
        if (cmin < mn) mn = cmin;
    }
    vector *com = node->get_com();
    node_rec r;
    r.level = level; r.count = count; r.min_index = mn; r.mass = node->get_mass();
    r.cx = com->get_x(); r.cy = com->get_y(); r.cz = com->get_z(); r.side = node->get_side();
    if (nchild < 2 && level != 0) r.level = -1; /* chain or empty node: dropped below */
    out[slot] = r;
    *min_index = mn;
    return count;
}

}  // namespace

extern "C" {

int ref_datatype_bytes(void) { return (int)sizeof(datatype); }

/* Seeded initial conditions in generation order (src/main.cpp:1379-1415). */
int ref_generate(const gen_params *g, unsigned int n, double *pos, double *vel, double *mass) {
    settings s;
    set_default(s);
    s.gen_type = (unsigned)g->gen_type;
    s.mass_dist = (unsigned)g->mass_dist;
    s.vel_dist = (unsigned)g->vel_dist;
    s.size = (datatype)g->size;
    s.min_mass = (datatype)g->min_mass;
    s.max_mass = (datatype)g->max_mass;
    s.min_vel = (datatype)g->min_vel;
    s.max_vel = (datatype)g->max_vel;
    s.r_sphere = (datatype)g->r_sphere;
    s.rotation_magnitude = (datatype)g->rotation_magnitude;
    s.rotation_vector = vector((datatype)g->rot_x, (datatype)g->rot_y, (datatype)g->rot_z);
    s.scale_x = (datatype)g->scale_x;
    s.scale_y = (datatype)g->scale_y;
    s.scale_z = (datatype)g->scale_z;
    std::default_random_engine generator;
    generator.seed(g->seed);
    for (unsigned int i = 0; i < n; i++) {
        particle_set one;
        generate_particle(s, &one, generator);
        particle *p = *one.begin();
        pos[3 * i] = p->get_pos()->get_x();
        pos[3 * i + 1] = p->get_pos()->get_y();
        pos[3 * i + 2] = p->get_pos()->get_z();
        vel[3 * i] = p->get_vel()->get_x();
        vel[3 * i + 1] = p->get_vel()->get_y();
        vel[3 * i + 2] = p->get_vel()->get_z();
        mass[i] = p->get_mass();
        delete p;
    }
    return 0;
}

/* One force pass: tree + mass/COM + barnes_hut_threaded. acc_out in input order.
 * times_out (optional, 3 doubles): build, mass+com, walk seconds. */
int ref_forces(unsigned int n, const double *pos, const double *mass, double theta, int damping,
               unsigned int threads, double *acc_out, double *times_out) {
    if (n == 0) return 0;
    std::vector<particle *> order;
    particle_set set;
    make_particles(n, pos, NULL, mass, order, set);
    settings cfg;
    settings_for_walk(cfg, theta, damping, threads);
    double tb = 0, tm = 0;
    octree *root = build_tree(&set, cfg.threads, &tb, &tm);
    double t0 = now_s();
    barnes_hut_threaded(cfg, &set, root, NULL, NULL);
    double tw = now_s() - t0;
    delete_tree(root, cfg.threads);
    for (unsigned int i = 0; i < n; i++) {
        vector *a = order[i]->get_acc();
        acc_out[3 * i] = a->get_x();
        acc_out[3 * i + 1] = a->get_y();
        acc_out[3 * i + 2] = a->get_z();
    }
    if (times_out) { times_out[0] = tb; times_out[1] = tm; times_out[2] = tw; }
    free_particles(order);
    return 0;
}

/* Tree over all n particles, walk for the `m` particles listed in `sample`
 * only (the reference walk takes the particle set and the root separately,
 * src/main.cpp:432). acc_out is m x 3. times_out as in ref_forces. */
int ref_forces_sample(unsigned int n, const double *pos, const double *mass, double theta,
                      int damping, unsigned int threads, const unsigned int *sample,
                      unsigned int m, double *acc_out, double *times_out) {
    if (n == 0) return 0;
    std::vector<particle *> order;
    particle_set set;
    make_particles(n, pos, NULL, mass, order, set);
    settings cfg;
    settings_for_walk(cfg, theta, damping, threads);
    double tb = 0, tm = 0;
    octree *root = build_tree(&set, cfg.threads, &tb, &tm);
    particle_set subset;
    subset.reserve(m);
    for (unsigned int i = 0; i < m; i++) subset.insert(order[sample[i]]);
    double t0 = now_s();
    barnes_hut_threaded(cfg, &subset, root, NULL, NULL);
    double tw = now_s() - t0;
    delete_tree(root, cfg.threads);
    for (unsigned int i = 0; i < m; i++) {
        vector *a = order[sample[i]]->get_acc();
        acc_out[3 * i] = a->get_x();
        acc_out[3 * i + 1] = a->get_y();
        acc_out[3 * i + 2] = a->get_z();
    }
    if (times_out) { times_out[0] = tb; times_out[1] = tm; times_out[2] = tw; }
    free_particles(order);
    return 0;
}

/* The frame loop of main() restricted to the hot path (src/main.cpp:1420-1492
 * with collide, min_node_size and dumps off). pos/vel are updated in place.
 * frames_out (optional) receives positions after every frame: frames x n x 3. */
int ref_run_frames(unsigned int n, double *pos, double *vel, const double *mass, double theta,
                   int damping, double dt, unsigned int threads, unsigned int frames,
                   double *frames_out) {
    if (n == 0) return 0;
    std::vector<particle *> order;
    particle_set set;
    make_particles(n, pos, vel, mass, order, set);
    settings cfg;
    settings_for_walk(cfg, theta, damping, threads);
    cfg.dt = (datatype)dt;
    for (unsigned int f = 0; f < frames; f++) {
        octree *root = build_tree(&set, cfg.threads, NULL, NULL);
        barnes_hut_threaded(cfg, &set, root, NULL, NULL);
        delete_tree(root, cfg.threads);
        if (cfg.threads > 1) update_all_threaded(cfg, &set);
        else update_all(cfg, &set);
        if (frames_out) {
            double *o = frames_out + (size_t)f * n * 3;
            for (unsigned int i = 0; i < n; i++) {
                o[3 * i] = order[i]->get_pos()->get_x();
                o[3 * i + 1] = order[i]->get_pos()->get_y();
                o[3 * i + 2] = order[i]->get_pos()->get_z();
            }
        }
    }
    for (unsigned int i = 0; i < n; i++) {
        pos[3 * i] = order[i]->get_pos()->get_x();
        pos[3 * i + 1] = order[i]->get_pos()->get_y();
        pos[3 * i + 2] = order[i]->get_pos()->get_z();
        vel[3 * i] = order[i]->get_vel()->get_x();
        vel[3 * i + 1] = order[i]->get_vel()->get_y();
        vel[3 * i + 2] = order[i]->get_vel()->get_z();
    }
    free_particles(order);
    return 0;
}

/* One frame of main()'s loop with the merging steps on (src/main.cpp:1420-1492,
 * serial build): gen_root -> apply_minimum_size (when min_size > 0) -> calc_mass
 * -> calc_com -> barnes_hut_threaded with collision capture (when collide) ->
 * update_collision -> update_all. The surviving particles come back in the
 * particle set's iteration order (n_out of them; at most cap are written):
 * position, velocity, acceleration and mass. Particles the reference erases
 * without deleting (apply_minimum_size) are left allocated: test use only. */
int ref_frame_merging(unsigned int n, const double *pos, const double *vel, const double *mass, double theta,
                      int damping, double dt, int collide, double collision_range, double min_size,
                      unsigned int cap, unsigned int *n_out, double *pos_out, double *vel_out, double *acc_out,
                      double *mass_out) {
    std::vector<particle *> order;
    particle_set *set = new particle_set;
    make_particles(n, pos, vel, mass, order, *set);
    settings cfg;
    settings_for_walk(cfg, theta, damping, 1);
    cfg.dt = (datatype)dt;
    cfg.collide = collide != 0;
    cfg.collision_range = (datatype)collision_range;
    cfg.min_node_size = (datatype)min_size;
    if (n > 0) {
        octree *root = gen_root(set);
        if (cfg.min_node_size > 0.0) apply_minimum_size(cfg.min_node_size, root, set, NULL);
        root->calc_mass();
        root->calc_com();
        particle_set *added = NULL, *removed = NULL;
        if (cfg.collide) {
            added = new particle_set;
            removed = new particle_set;
        }
        barnes_hut_threaded(cfg, set, root, added, removed);
        delete root;
        if (cfg.collide) {
            update_collision(set, added, removed, false);
            delete added;
            delete removed;
        }
        update_all(cfg, set);
    }
    unsigned int k = 0;
    for (particle_set::iterator it = set->begin(); it != set->end(); ++it, ++k) {
        if (k >= cap) continue;
        particle *q = *it;
        pos_out[3 * k] = q->get_pos()->get_x(); pos_out[3 * k + 1] = q->get_pos()->get_y();
        pos_out[3 * k + 2] = q->get_pos()->get_z();
        vel_out[3 * k] = q->get_vel()->get_x(); vel_out[3 * k + 1] = q->get_vel()->get_y();
        vel_out[3 * k + 2] = q->get_vel()->get_z();
        acc_out[3 * k] = q->get_acc()->get_x(); acc_out[3 * k + 1] = q->get_acc()->get_y();
        acc_out[3 * k + 2] = q->get_acc()->get_z();
        mass_out[k] = q->get_mass();
    }
    *n_out = k;
    for (particle_set::iterator it = set->begin(); it != set->end(); ++it) delete *it;
    delete set;
    return 0;
}

/* The reference's write_image (src/main.cpp:556-678) on n positions; the
 * rendered 24-bit bitmap comes back through the FreeImage stand-in:
 * rgb_out[(y * w + x) * 3 + {R, G, B}], y as FreeImage counts it (row 0 at the
 * bottom of the saved image). Returns 0 on success. */
int ref_write_image(unsigned int n, const double *pos, unsigned int img_w, unsigned int img_h,
                    unsigned int projection, unsigned int color, int adaptive, int nonlinear, double scale,
                    double brightness, unsigned char *rgb_out) {
    std::vector<particle *> order;
    particle_set set;
    std::vector<double> mass(n, 1.0);
    make_particles(n, pos, NULL, mass.data(), order, set);
    g_stub_last_image = FIBITMAP{0, 0, std::vector<unsigned char>()};
    write_image(img_w, img_h, projection, color, adaptive != 0, nonlinear != 0, (datatype)scale,
                (datatype)brightness, 0, &set);
    free_particles(order);
    if (g_stub_last_image.w != (int)img_w || g_stub_last_image.h != (int)img_h) return -1;
    std::memcpy(rgb_out, g_stub_last_image.rgb.data(), g_stub_last_image.rgb.size());
    return 0;
}

/* The reference's unmodified main() (src/main.cpp:1359-1504), for running the
 * whole program in-process: argv[1] is a settings file; output goes to ./data. */
int ref_main(int argc, char **argv) { return nbodysim_reference_main(argc, argv); }

/* Branching nodes of the reference tree (nodes with >= 2 non-empty children,
 * plus the root), pre-order. Each record: level, particle count, smallest
 * input index inside, mass, com, side. Returns the record count (or the
 * required count when it exceeds cap); *depth_out gets the deepest level. */
int ref_tree_nodes(unsigned int n, const double *pos, const double *mass, unsigned int threads,
                   int cap, int *level, int *count, int *min_index, double *node_mass,
                   double *com, double *side, int *depth_out) {
    if (n == 0) return 0;
    std::vector<particle *> order;
    particle_set set;
    make_particles(n, pos, NULL, mass, order, set);
    octree *root = build_tree(&set, threads ? threads : 1, NULL, NULL);
    std::unordered_map<particle *, int> index;
    for (unsigned int i = 0; i < n; i++) index[order[i]] = (int)i;
    std::vector<node_rec> out;
    int mn = 0, depth = 0;
    collect(root, 0, index, out, &mn, &depth);
    delete_tree(root, threads ? threads : 1);
    size_t kept = 0;
    for (size_t i = 0; i < out.size(); i++)
        if (out[i].level >= 0) out[kept++] = out[i];
    out.resize(kept);
    free_particles(order);
    if (depth_out) *depth_out = depth;
    if ((int)out.size() > cap) return (int)out.size();
    for (size_t i = 0; i < out.size(); i++) {
        level[i] = out[i].level; count[i] = out[i].count; min_index[i] = out[i].min_index;
        node_mass[i] = out[i].mass; side[i] = out[i].side;
        com[3 * i] = out[i].cx; com[3 * i + 1] = out[i].cy; com[3 * i + 2] = out[i].cz;
    }
    return (int)out.size();
}

}  // extern "C"
