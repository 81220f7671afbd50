// capi.cu -- extern "C" entry points of include/dmdgpu.h.
//
// No C++ exception crosses this boundary: every entry point returns a status
// code and leaves a message retrievable with dmdgpu_last_error.
#include <cuda_runtime.h>

#include <cstring>
#include <memory>
#include <new>
#include <string>

#include "engine.h"

struct dmdgpu_ctx {
    std::unique_ptr<dmd::Batch> b;
    int slot = -1;
    dmdgpu_options opt{};
    std::string err;
};

struct dmdgpu_batch {
    std::unique_ptr<dmd::Batch> b;
    std::string err;
};

namespace {

int ctx_fail(dmdgpu_ctx* c, int code) {
    if (c && c->b) c->err = c->b->error();
    return code;
}

// A dmdgpu_system view of a host system (positions / box optionally replaced).
struct SysView {
    dmdgpu_system s{};
};

SysView view_of(const dmd::HostSystem& h, const double* x, const double* y, const double* z,
                double box, unsigned mask) {
    SysView v;
    dmdgpu_system& s = v.s;
    s.n_atoms = h.n;
    s.box_size = box;
    s.masses = h.mass.data();
    s.charges = h.q.data();
    s.pos_x = x;
    s.pos_y = y;
    s.pos_z = z;
    s.vel_x = h.vx.data();
    s.vel_y = h.vy.data();
    s.vel_z = h.vz.data();
    s.atom_types = h.type.data();
    s.use_lj = h.use_lj;
    s.lj_n_types = h.n_types;
    s.lj_sigma = h.sigma.data();
    s.lj_epsilon = h.eps.data();
    s.lj_cutoff = h.lj_cutoff;
    if (mask & dmd::C_BOND) {
        s.n_bonds = static_cast<int>(h.bi.size());
        s.bond_i = h.bi.data();
        s.bond_j = h.bj.data();
        s.bond_k = h.bk.data();
        s.bond_r0 = h.br0.data();
    }
    if (mask & dmd::C_ANGLE) {
        s.n_angles = static_cast<int>(h.ai.size());
        s.angle_i = h.ai.data();
        s.angle_j = h.aj.data();
        s.angle_k = h.ak.data();
        s.angle_k_theta = h.akt.data();
        s.angle_theta0 = h.at0.data();
    }
    if (mask & dmd::C_DIH) {
        s.n_dihedrals = static_cast<int>(h.di.size());
        s.dihedral_i = h.di.data();
        s.dihedral_j = h.dj.data();
        s.dihedral_k = h.dk.data();
        s.dihedral_l = h.dl.data();
        s.dihedral_periodicity = h.dn.data();
        s.dihedral_k_phi = h.dkp.data();
        s.dihedral_phi0 = h.dp0.data();
    }
    if (mask & dmd::C_IMP) {
        s.n_impropers = static_cast<int>(h.ii.size());
        s.improper_i = h.ii.data();
        s.improper_j = h.ij.data();
        s.improper_k = h.ik.data();
        s.improper_l = h.il.data();
        s.improper_k_phi = h.ikp.data();
        s.improper_phi0 = h.ip0.data();
    }
    s.coulomb_type = h.coulomb_type;
    s.coulomb_cutoff = h.coul_cutoff;
    s.ewald_coeff = h.ewald;
    s.pme_grid_spacing = h.spacing;
    s.pme_order = h.pme_order;
    s.n_excl = static_cast<int>(h.ei.size());
    s.excl_i = h.ei.data();
    s.excl_j = h.ej.data();
    s.dt = h.dt;
    s.n_steps = h.n_steps;
    return v;
}

}  // namespace

extern "C" {

int dmdgpu_create(const dmdgpu_system* sys, const dmdgpu_options* opt, dmdgpu_ctx** out) {
    if (!out) return DMDGPU_ERR_INVALID;
    *out = nullptr;
    if (!sys || !opt) return DMDGPU_ERR_INVALID;
    auto* c = new (std::nothrow) dmdgpu_ctx();
    if (!c) return DMDGPU_ERR_OOM;
    *out = c;
    c->opt = *opt;
    try {
        c->b = std::make_unique<dmd::Batch>(*opt, 0);
    } catch (const std::exception& e) {
        c->err = e.what();
        return DMDGPU_ERR_GPU;
    }
    int slot = -1;
    int rc = c->b->add(*sys, 0, dmd::C_ALL, &slot);
    if (rc) return ctx_fail(c, rc);
    c->slot = slot;
    rc = c->b->pack();
    if (rc) return ctx_fail(c, rc);
    return DMDGPU_OK;
}

int dmdgpu_step(dmdgpu_ctx* c, int32_t n) {
    if (!c || !c->b) return DMDGPU_ERR_INVALID;
    if (n < 0) return DMDGPU_ERR_PARM;
    int rc = c->b->extend_targets(n);
    if (!rc) rc = c->b->step(n);
    return rc ? ctx_fail(c, rc) : DMDGPU_OK;
}

int dmdgpu_run(dmdgpu_ctx* c) {
    if (!c || !c->b) return DMDGPU_ERR_INVALID;
    const dmd::HostSystem& h = c->b->system(c->slot);
    const int total = h.n_steps, every = h.checkpoint_interval;
    const bool ckpt = every > 0 && !h.checkpoint_path.empty();
    const std::string path = h.checkpoint_path;
    int done = 0;
    while (done < total) {
        int take = total - done;
        dmdgpu_scalars s;
        int rc = c->b->get_scalars(c->slot, &s);
        if (rc) return ctx_fail(c, rc);
        if (ckpt) {
            const long long to_next = every - (s.step % every);
            if (to_next < take) take = static_cast<int>(to_next);
        }
        rc = dmdgpu_step(c, take);
        if (rc) return rc;
        done += take;
        if (ckpt) {
            rc = c->b->get_scalars(c->slot, &s);
            if (!rc && s.step % every == 0) rc = c->b->save_checkpoint(c->slot, path.c_str());
            if (rc) return ctx_fail(c, rc);
        }
    }
    return DMDGPU_OK;
}

int dmdgpu_get_state(dmdgpu_ctx* c, int32_t which, double* x, double* y, double* z) {
    if (!c || !c->b || !x || !y || !z) return DMDGPU_ERR_INVALID;
    int rc = c->b->get_state(c->slot, which, x, y, z);
    return rc ? ctx_fail(c, rc) : DMDGPU_OK;
}

int dmdgpu_set_state(dmdgpu_ctx* c, int32_t which, const double* x, const double* y, const double* z) {
    if (!c || !c->b || !x || !y || !z) return DMDGPU_ERR_INVALID;
    int rc = c->b->set_state(c->slot, which, x, y, z);
    return rc ? ctx_fail(c, rc) : DMDGPU_OK;
}

int dmdgpu_get_scalars(dmdgpu_ctx* c, dmdgpu_scalars* out) {
    if (!c || !c->b || !out) return DMDGPU_ERR_INVALID;
    int rc = c->b->get_scalars(c->slot, out);
    return rc ? ctx_fail(c, rc) : DMDGPU_OK;
}

int dmdgpu_compute_forces(dmdgpu_ctx* c, double* fx, double* fy, double* fz, double* e_terms) {
    if (!c || !c->b) return DMDGPU_ERR_INVALID;
    int rc = c->b->compute_forces(c->slot, fx, fy, fz, e_terms);
    return rc ? ctx_fail(c, rc) : DMDGPU_OK;
}

int dmdgpu_component_compute(dmdgpu_ctx* c, int32_t component, const double* px, const double* py,
                             const double* pz, double box, double* fx, double* fy, double* fz,
                             double* energy) {
    if (!c || !c->b || !px || !py || !pz || !fx || !fy || !fz || !energy) return DMDGPU_ERR_INVALID;
    static const unsigned masks[8] = {dmd::C_LJ, dmd::C_BOND, dmd::C_ANGLE, dmd::C_DIH, dmd::C_CREAL,
                                      dmd::C_PME, dmd::C_EXCL, dmd::C_IMP};
    if (component < 0 || component > 7) {
        c->err = "component must be 0..7";
        return DMDGPU_ERR_PARM;
    }
    const dmd::HostSystem& h = c->b->system(c->slot);
    const unsigned mask = masks[component];
    SysView v = view_of(h, px, py, pz, box, mask);
    // evaluate on a scratch table so the context's own state is untouched
    try {
        dmd::Batch tmp(c->opt, 0);
        int slot = -1;
        int arc = tmp.add(v.s, 0, mask, &slot);
        if (arc) {
            c->err = tmp.error();
            return arc;
        }
        const int n = h.n;
        std::vector<double> gx(n), gy(n), gz(n);
        double e[9];
        int rc = tmp.compute_forces(slot, gx.data(), gy.data(), gz.data(), e);
        if (rc) {
            c->err = tmp.error();
            return rc;
        }
        for (int i = 0; i < n; ++i) {
            fx[i] += gx[i];
            fy[i] += gy[i];
            fz[i] += gz[i];
        }
        static const int term[8][2] = {{0, -1}, {5, -1}, {6, -1}, {7, -1}, {1, -1}, {2, 3}, {4, -1}, {8, -1}};
        double add = e[term[component][0]];
        if (term[component][1] >= 0) add += e[term[component][1]];
        *energy += add;
    } catch (const std::exception& ex) {
        c->err = ex.what();
        return DMDGPU_ERR_GPU;
    }
    return DMDGPU_OK;
}

int dmdgpu_pair_list(dmdgpu_ctx* c, int32_t* pi, int32_t* pj, int64_t cap, int64_t* count) {
    if (!c || !c->b || !count) return DMDGPU_ERR_INVALID;
    long long cnt = 0;
    int rc = c->b->pair_list(c->slot, pi, pj, (pi && pj) ? cap : 0, &cnt);
    *count = cnt;
    return rc ? ctx_fail(c, rc) : DMDGPU_OK;
}

int dmdgpu_save_checkpoint(dmdgpu_ctx* c, const char* path) {
    if (!c || !c->b || !path) return DMDGPU_ERR_INVALID;
    int rc = c->b->save_checkpoint(c->slot, path);
    return rc ? ctx_fail(c, rc) : DMDGPU_OK;
}

int dmdgpu_load_checkpoint(dmdgpu_ctx* c, const char* path) {
    if (!c || !c->b || !path) return DMDGPU_ERR_INVALID;
    int rc = c->b->load_checkpoint(c->slot, path);
    return rc ? ctx_fail(c, rc) : DMDGPU_OK;
}

int64_t dmdgpu_footprint_bytes(const dmdgpu_system* sys, const dmdgpu_options* opt) {
    if (!sys || !opt) return -1;
    dmd::HostSystem h;
    h.n = sys->n_atoms;
    h.box = sys->box_size;
    h.coulomb_type = sys->coulomb_type;
    h.spacing = sys->pme_grid_spacing;
    try {
        dmd::Batch tmp(*opt, 0);
        return tmp.footprint(h);
    } catch (...) {
        return -1;
    }
}

int dmdgpu_repack(dmdgpu_ctx* c) {
    if (!c || !c->b) return DMDGPU_ERR_INVALID;
    int rc = c->b->repack();
    return rc ? ctx_fail(c, rc) : DMDGPU_OK;
}

int64_t dmdgpu_kernel_launches(dmdgpu_ctx* c) { return (c && c->b) ? c->b->launches() : 0; }

void* dmdgpu_stream(dmdgpu_ctx* c) { return (c && c->b) ? static_cast<void*>(c->b->stream()) : nullptr; }

int dmdgpu_get_launch_info(dmdgpu_ctx* c, dmdgpu_launch_info* out) {
    if (!c || !c->b || !out) return DMDGPU_ERR_INVALID;
    c->b->launch_info(out);
    return DMDGPU_OK;
}

int dmdgpu_step_timed(dmdgpu_ctx* c, int32_t n, int64_t flush_bytes, dmdgpu_timing* out) {
    if (!c || !c->b || n <= 0 || !out) return DMDGPU_ERR_INVALID;
    int rc = c->b->extend_targets(n);
    if (!rc) rc = c->b->step_timed(n, flush_bytes, out);
    return rc ? ctx_fail(c, rc) : DMDGPU_OK;
}

int dmdgpu_set_frame_writer(dmdgpu_ctx* c, int32_t interval, dmdgpu_frame_fn fn, void* user) {
    if (!c || !c->b) return DMDGPU_ERR_INVALID;
    int rc = c->b->set_frame_writer(interval, fn, user);
    return rc ? ctx_fail(c, rc) : DMDGPU_OK;
}

int dmdgpu_flush_frames(dmdgpu_ctx* c) {
    if (!c || !c->b) return DMDGPU_ERR_INVALID;
    int rc = c->b->flush_frames();
    return rc ? ctx_fail(c, rc) : DMDGPU_OK;
}

int dmdgpu_test_inject(dmdgpu_ctx* c, int32_t what) {
    if (!c || !c->b) return DMDGPU_ERR_INVALID;
    int rc = c->b->inject(what);
    return rc ? ctx_fail(c, rc) : DMDGPU_OK;
}

const char* dmdgpu_last_error(const dmdgpu_ctx* c) { return c ? c->err.c_str() : "null context"; }

void dmdgpu_destroy(dmdgpu_ctx* c) { delete c; }

// ---- batch / serving ---------------------------------------------------------
int dmdgpu_batch_create(int64_t budget, const dmdgpu_options* opt, dmdgpu_batch** out) {
    if (!out || !opt) return DMDGPU_ERR_INVALID;
    *out = nullptr;
    auto* b = new (std::nothrow) dmdgpu_batch();
    if (!b) return DMDGPU_ERR_OOM;
    *out = b;
    try {
        b->b = std::make_unique<dmd::Batch>(*opt, budget);
    } catch (const std::exception& e) {
        b->err = e.what();
        return DMDGPU_ERR_GPU;
    }
    return DMDGPU_OK;
}

int dmdgpu_batch_admit(dmdgpu_batch* b, const dmdgpu_system* sys, int64_t n_steps, int32_t* slot) {
    if (!b || !b->b || !sys || !slot) return DMDGPU_ERR_INVALID;
    int s = -1;
    int rc = b->b->add(*sys, n_steps, dmd::C_ALL, &s);
    if (rc) {
        b->err = b->b->error();
        return rc;
    }
    *slot = s;
    return DMDGPU_OK;
}

int dmdgpu_batch_step(dmdgpu_batch* b, int32_t n) {
    if (!b || !b->b) return DMDGPU_ERR_INVALID;
    int rc = b->b->step(n);
    if (rc) b->err = b->b->error();
    return rc;
}

int dmdgpu_batch_step_timed(dmdgpu_batch* b, int32_t n, int64_t flush_bytes, dmdgpu_timing* out) {
    if (!b || !b->b || n <= 0 || !out) return DMDGPU_ERR_INVALID;
    int rc = b->b->step_timed(n, flush_bytes, out);
    if (rc) b->err = b->b->error();
    return rc;
}

int dmdgpu_batch_poll(dmdgpu_batch* b, int32_t* slots, int32_t cap, int32_t* n_done) {
    if (!b || !b->b || !n_done) return DMDGPU_ERR_INVALID;
    int nd = 0;
    int rc = b->b->poll(slots, cap, &nd);
    *n_done = nd;
    return rc;
}

int dmdgpu_batch_get_state(dmdgpu_batch* b, int32_t slot, int32_t which, double* x, double* y, double* z) {
    if (!b || !b->b || !x || !y || !z) return DMDGPU_ERR_INVALID;
    int rc = b->b->get_state(slot, which, x, y, z);
    if (rc) b->err = b->b->error();
    return rc;
}

int dmdgpu_batch_get_scalars(dmdgpu_batch* b, int32_t slot, dmdgpu_scalars* out) {
    if (!b || !b->b || !out) return DMDGPU_ERR_INVALID;
    int rc = b->b->get_scalars(slot, out);
    if (rc) b->err = b->b->error();
    return rc;
}

int dmdgpu_batch_release(dmdgpu_batch* b, int32_t slot) {
    if (!b || !b->b) return DMDGPU_ERR_INVALID;
    int rc = b->b->release(slot);
    if (rc) b->err = b->b->error();
    return rc;
}

int64_t dmdgpu_batch_used_bytes(dmdgpu_batch* b) { return (b && b->b) ? b->b->used_bytes() : 0; }

int dmdgpu_batch_get_launch_info(dmdgpu_batch* b, dmdgpu_launch_info* out) {
    if (!b || !b->b || !out) return DMDGPU_ERR_INVALID;
    b->b->launch_info(out);
    return DMDGPU_OK;
}

int32_t dmdgpu_batch_active(dmdgpu_batch* b) { return (b && b->b) ? b->b->active() : 0; }

const char* dmdgpu_batch_last_error(const dmdgpu_batch* b) { return b ? b->err.c_str() : "null batch"; }

void dmdgpu_batch_destroy(dmdgpu_batch* b) { delete b; }

}  // extern "C"
