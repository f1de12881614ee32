// extern "C" boundary: include/cgfdm.h.
#include "../../include/cgfdm.h"

#include <cuda_runtime.h>

#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "batch.hpp"
#include "session.hpp"

struct cgfdm_session {
    cgfdm::Session s;
};

struct cgfdm_batch {
    cgfdm::Batch b;
};

static thread_local std::string g_create_error;

#ifndef CGFDM_FLAVOR
#define CGFDM_FLAVOR "fast"
#endif

extern "C" {

const char *cgfdm_build_flavor(void) { return CGFDM_FLAVOR; }

int cgfdm_create(const char *run_dir, const char *options_json, int device, cgfdm_session **out)
{
    if (!run_dir || !out) {
        g_create_error = "run_dir and out must not be NULL";
        return CGFDM_E_ARG;
    }
    *out = nullptr;
    cgfdm_session *h = new (std::nothrow) cgfdm_session;
    if (!h) {
        g_create_error = "out of host memory";
        return CGFDM_E_ALLOC;
    }
    int st = h->s.create(run_dir, options_json ? options_json : "", device);
    if (st) {
        g_create_error = h->s.err;
        delete h;
        return st;
    }
    *out = h;
    return CGFDM_OK;
}

int cgfdm_create_part(const char *run_dir, const char *options_json, const int *parts, const int *coord, int device,
                      cgfdm_session **out)
{
    if (!run_dir || !out || !parts || !coord) {
        g_create_error = "run_dir, parts, coord and out must not be NULL";
        return CGFDM_E_ARG;
    }
    *out = nullptr;
    cgfdm_session *h = new (std::nothrow) cgfdm_session;
    if (!h) {
        g_create_error = "out of host memory";
        return CGFDM_E_ALLOC;
    }
    int st = h->s.create_part(run_dir, options_json ? options_json : "", parts, coord, device);
    if (st) {
        g_create_error = h->s.err;
        delete h;
        return st;
    }
    *out = h;
    return CGFDM_OK;
}

int cgfdm_part_info(const cgfdm_session *s, int *lo, int *n, int *top)
{
    if (!s) return CGFDM_E_ARG;
    const cgfdm::Model &m = s->s.m;
    if (lo) lo[0] = m.part_lo[0], lo[1] = m.part_lo[1], lo[2] = m.part_lo[2];
    if (n) n[0] = m.g.nx, n[1] = m.g.ny, n[2] = m.g.nz;
    if (top) *top = m.fs_top ? 1 : 0;
    return CGFDM_OK;
}

int cgfdm_part_station_ids(const cgfdm_session *s, int *ids, int count)
{
    if (!s || (!ids && count)) return CGFDM_E_ARG;
    const std::vector<int> &v = s->s.m.station_ids;
    if (count < (int)v.size()) return CGFDM_E_ARG;
    for (size_t i = 0; i < v.size(); i++) ids[i] = v[i];
    return CGFDM_OK;
}

int cgfdm_part_advance(cgfdm_session *s, int *phase)
{
    if (!s) return CGFDM_E_ARG;
    return s->s.part_advance(phase);
}

int cgfdm_part_launch(cgfdm_session *s, int *phase)
{
    if (!s) return CGFDM_E_ARG;
    return s->s.part_launch(phase);
}

int cgfdm_part_finish(cgfdm_session *s)
{
    if (!s) return CGFDM_E_ARG;
    return s->s.part_finish();
}

int cgfdm_part_link(cgfdm_session *s, int face, const cgfdm_session *nbr)
{
    if (!s || !nbr) return CGFDM_E_ARG;
    return s->s.link_halo(face, nbr->s);
}

int cgfdm_part_handle(cgfdm_session *s, void *out, long long bytes)
{
    if (!s) return CGFDM_E_ARG;
    return s->s.part_handle(out, bytes);
}

int cgfdm_part_link_handle(cgfdm_session *s, int face, const void *handle, long long bytes)
{
    if (!s) return CGFDM_E_ARG;
    return s->s.link_halo_handle(face, handle, bytes);
}

long long cgfdm_halo_count(const cgfdm_session *s, int face, int which)
{
    if (!s) return -1;
    return s->s.halo_count(face, which);
}

int cgfdm_halo_pack(cgfdm_session *s, int face, int which, float *d_buf)
{
    if (!s) return CGFDM_E_ARG;
    return s->s.halo_copy(face, which, d_buf, true);
}

int cgfdm_halo_unpack(cgfdm_session *s, int face, int which, const float *d_buf)
{
    if (!s) return CGFDM_E_ARG;
    return s->s.halo_copy(face, which, const_cast<float *>(d_buf), false);
}

int cgfdm_model_medium(const char *run_dir, const char *options_json, float *out, long long count, int *dims)
{
    if (!run_dir) {
        g_create_error = "run_dir must not be NULL";
        return CGFDM_E_ARG;
    }
    cgfdm::Model m;
    std::string err;
    int st = cgfdm::build_model(run_dir, options_json ? options_json : "", m, err);
    if (st) {
        g_create_error = err;
        return st;
    }
    if (dims) dims[0] = m.g._nz_, dims[1] = m.g._ny_, dims[2] = m.g._nx_;
    if (!out) return CGFDM_OK;
    if (count < (long long)m.medium.size()) {
        g_create_error = "output array too small for the medium";
        return CGFDM_E_ARG;
    }
    std::memcpy(out, m.medium.data(), sizeof(float) * m.medium.size());
    return CGFDM_OK;
}

int cgfdm_model_coord(const char *run_dir, const char *options_json, float *terrain, long long terrain_count,
                      float *coord, long long coord_count, int *dims)
{
    if (!run_dir) {
        g_create_error = "run_dir must not be NULL";
        return CGFDM_E_ARG;
    }
    cgfdm::Model m;
    std::string err;
    int st = cgfdm::build_model(run_dir, options_json ? options_json : "", m, err);
    if (st) {
        g_create_error = err;
        return st;
    }
    if (dims) dims[0] = m.g._nz_, dims[1] = m.g._ny_, dims[2] = m.g._nx_;
    if (coord) cgfdm::materialize_coords(m);
    if ((terrain && terrain_count < (long long)m.terrain.size()) || (coord && coord_count < (long long)m.coord.size())) {
        g_create_error = "output array too small";
        return CGFDM_E_ARG;
    }
    if (terrain) std::memcpy(terrain, m.terrain.data(), sizeof(float) * m.terrain.size());
    if (coord) std::memcpy(coord, m.coord.data(), sizeof(float) * m.coord.size());
    return CGFDM_OK;
}

int cgfdm_check_finite(cgfdm_session *s, long long *count, long long *first)
{
    if (!s) return CGFDM_E_ARG;
    return s->s.check_finite(count, first);
}

int cgfdm_run(cgfdm_session *s, int nsteps)
{
    if (!s) return CGFDM_E_ARG;
    return s->s.run(nsteps);
}

int cgfdm_run_timed(cgfdm_session *s, int nsteps, float *ms)
{
    if (!s || !ms) return CGFDM_E_ARG;
    return s->s.run_timed(nsteps, ms, nullptr);
}

int cgfdm_info_get(const cgfdm_session *s, cgfdm_info *o)
{
    if (!s || !o) return CGFDM_E_ARG;
    const auto &S = s->s;
    std::memset(o, 0, sizeof *o);
    o->scheme = S.m.p.scheme;
    o->nx = S.m.g.nx, o->ny = S.m.g.ny, o->nz = S.m.g.nz;
    o->nxp = S.m.g._nx_, o->nyp = S.m.g._ny_, o->nzp = S.m.g._nz_;
    o->NT = S.m.NT;
    o->steps_done = S.it;
    o->n_stations = S.nst;
    o->n_fault_cells = S.m.fault.npts;
    o->DT = (float)S.m.p.DT;
    o->DH = S.m.g.DH;
    o->dtmax = S.m.dtmax;
    o->H_min = S.m.H_min;
    o->Vp_max = S.m.Vp_max;
    o->device_bytes = (double)S.device_bytes;
    o->h2d_bytes = S.h2d_bytes;
    o->kernel_launches = S.kernel_launches;
    o->algo_bytes_per_step = S.algo_bytes_per_step();
    o->stage_kernels_per_step = S.m.p.scheme == 0 ? 4 : 3;
    o->pgv_fields = S.pgv_fields();
    return CGFDM_OK;
}

int cgfdm_create_profile(const cgfdm_session *s, double *ms)
{
    if (!s || !ms) return CGFDM_E_ARG;
    for (int i = 0; i < 3; i++) ms[i] = s->s.create_ms[i];
    ms[3] = s->s.capture_ms;
    for (int i = 0; i < 5; i++) ms[4 + i] = s->s.m.phase_ms[i];
    for (int i = 0; i < 5; i++) ms[9 + i] = s->s.setup_ms[i];
    return CGFDM_OK;
}

int cgfdm_profile_stages(cgfdm_session *s, int nsteps, float *mean_stage_ms)
{
    if (!s || !mean_stage_ms || nsteps <= 0) return CGFDM_E_ARG;
    return s->s.profile_stages(nsteps, mean_stage_ms);
}

int cgfdm_get_stations(const cgfdm_session *s, float *out, long long count)
{
    if (!s || (!out && s->s.nst > 0)) return CGFDM_E_ARG;
    if (count < (long long)s->s.nst * s->s.m.NT * 9) return CGFDM_E_ARG;
    return s->s.get_stations(out);
}

int cgfdm_get_wavefield(const cgfdm_session *s, float *out, long long count)
{
    if (!s || !out) return CGFDM_E_ARG;
    if (count < s->s.m.g.npad() * 9) return CGFDM_E_ARG;
    return s->s.get_wavefield(out);
}

int cgfdm_get_cjm(const cgfdm_session *s, float *out, long long count, int *nfield)
{
    if (!s) return CGFDM_E_ARG;
    int nf = 0;
    s->s.get_cjm(nullptr, &nf);
    if (nfield) *nfield = nf;
    if (!out) return CGFDM_OK;
    if (count < s->s.m.g.npad() * nf) return CGFDM_E_ARG;
    return s->s.get_cjm(out, nullptr);
}

int cgfdm_get_pgv(const cgfdm_session *s, float *out, long long count)
{
    if (!s || !out) return CGFDM_E_ARG;
    if (count < (long long)s->s.m.g.nx * s->s.m.g.ny * s->s.pgv_fields()) return CGFDM_E_ARG;
    return s->s.get_pgv(out);
}

int cgfdm_get_array(cgfdm_session *s, const char *name, void *out, long long *bytes)
{
    if (!s || !name || !bytes) return CGFDM_E_ARG;
    return s->s.get_array(name, out, bytes);
}

int cgfdm_write_outputs(const cgfdm_session *s)
{
    if (!s) return CGFDM_E_ARG;
    return s->s.write_outputs();
}

int cgfdm_checkpoint_size(const cgfdm_session *s, long long *bytes)
{
    if (!s || !bytes) return CGFDM_E_ARG;
    *bytes = (long long)s->s.checkpoint_bytes();
    return CGFDM_OK;
}

int cgfdm_checkpoint(cgfdm_session *s, void *out, long long bytes)
{
    if (!s || !out || bytes < 0) return CGFDM_E_ARG;
    return s->s.checkpoint(out, (size_t)bytes);
}

int cgfdm_restore(cgfdm_session *s, const void *in, long long bytes)
{
    if (!s || !in || bytes < 0) return CGFDM_E_ARG;
    return s->s.restore(in, (size_t)bytes);
}

int cgfdm_set_wavefield(cgfdm_session *s, const float *in, long long count)
{
    if (!s || !in) return CGFDM_E_ARG;
    if (count < s->s.m.g.npad() * 9) return CGFDM_E_ARG;
    return s->s.set_wavefield(in);
}

int cgfdm_set_medium(cgfdm_session *s, const float *medium, long long count)
{
    if (!s || !medium) return CGFDM_E_ARG;
    if (count < s->s.m.g.npad() * 3) return CGFDM_E_ARG;
    return s->s.set_medium(medium);
}

int cgfdm_adjoint_apply(cgfdm_session *s, int nsteps, float *state, long long count)
{
    if (!s || !state) return CGFDM_E_ARG;
    if (count < s->s.m.g.npad() * 9) return CGFDM_E_ARG;
    return s->s.adjoint_apply(nsteps, state);
}

int cgfdm_gradient(cgfdm_session *s, const float *observed, long long obs_count, int checkpoint_every,
                   double *misfit, float *grad, long long grad_count)
{
    if (!s || !grad || (!observed && s->s.nst > 0)) return CGFDM_E_ARG;
    if (obs_count < (long long)s->s.nst * s->s.m.NT * 3) return CGFDM_E_ARG;
    if (grad_count < 3LL * s->s.m.g.nx * s->s.m.g.ny * s->s.m.g.nz) return CGFDM_E_ARG;
    return s->s.gradient(observed, checkpoint_every, misfit, grad);
}

int cgfdm_autotune(cgfdm_session *s, int trial_steps, int *kchunk, int *ctas, float *ms_per_step)
{
    if (!s || trial_steps < 1) return CGFDM_E_ARG;
    return s->s.autotune(trial_steps, kchunk, ctas, ms_per_step);
}

int cgfdm_run_precise(cgfdm_session *s, int nsteps, int bits, double *stations, long long n_stations,
                      double *pgv, long long n_pgv, double *wavefield, long long n_wavefield)
{
    if (!s) return CGFDM_E_ARG;
    const cgfdm::Model &m = s->s.m;
    const long long need_st = (long long)s->s.nst * nsteps * 9, need_pgv = (long long)m.g.nx * m.g.ny * 2;
    const long long need_w = m.g.npad() * 9;
    if ((stations && n_stations < need_st) || (pgv && n_pgv < need_pgv) || (wavefield && n_wavefield < need_w)) {
        s->s.err = "cgfdm_run_precise: output buffer too small";
        return CGFDM_E_ARG;
    }
    return s->s.run_precise(nsteps, bits, stations, pgv, wavefield);
}

int cgfdm_test_stall(cgfdm_session *s, int item, int fill, long long wait_cycles)
{
    if (!s) return CGFDM_E_ARG;
    return s->s.test_stall(item, fill, wait_cycles);
}

int cgfdm_set_tiling(cgfdm_session *s, int kchunk, int ctas)
{
    if (!s) return CGFDM_E_ARG;
    return s->s.set_tiling(kchunk, ctas);
}

int cgfdm_get_tiling(const cgfdm_session *s, int *kchunk, int *ctas)
{
    if (!s) return CGFDM_E_ARG;
    if (kchunk) *kchunk = s->s.kchunk();
    if (ctas) *ctas = s->s.ctas();
    return CGFDM_OK;
}

int cgfdm_set_stage_tile(cgfdm_session *s, int rows)
{
    if (!s) return CGFDM_E_ARG;
    return s->s.set_tile(rows);
}

int cgfdm_get_stage_tile(const cgfdm_session *s, int *rows)
{
    if (!s || !rows) return CGFDM_E_ARG;
    *rows = s->s.tile();
    return CGFDM_OK;
}

int cgfdm_batch_autotune(cgfdm_batch *b, int trial_steps, int *kchunk, int *ctas, float *ms_per_step)
{
    if (!b || trial_steps < 1) return CGFDM_E_ARG;
    return b->b.autotune(trial_steps, kchunk, ctas, ms_per_step);
}

int cgfdm_batch_set_stage_tile(cgfdm_batch *b, int rows)
{
    if (!b) return CGFDM_E_ARG;
    return b->b.set_tile(rows);
}

int cgfdm_batch_get_stage_tile(const cgfdm_batch *b, int *rows)
{
    if (!b || !rows) return CGFDM_E_ARG;
    *rows = b->b.tile();
    return CGFDM_OK;
}

int cgfdm_gradient_profile(const cgfdm_session *s, float *ms3)
{
    if (!s || !ms3) return CGFDM_E_ARG;
    for (int c = 0; c < 3; c++) ms3[c] = s->s.grad_ms[c];
    return CGFDM_OK;
}

int cgfdm_batch_create(cgfdm_session *const *sessions, int n, cgfdm_batch **out)
{
    if (!sessions || n <= 0 || !out) {
        g_create_error = "sessions, n > 0 and out are required";
        return CGFDM_E_ARG;
    }
    *out = nullptr;
    std::vector<cgfdm::Session *> v;
    for (int i = 0; i < n; i++) {
        if (!sessions[i]) {
            g_create_error = "NULL session in batch";
            return CGFDM_E_ARG;
        }
        v.push_back(&sessions[i]->s);
    }
    cgfdm_batch *h = new (std::nothrow) cgfdm_batch;
    if (!h) {
        g_create_error = "out of host memory";
        return CGFDM_E_ALLOC;
    }
    int st = h->b.create(v);
    if (st) {
        g_create_error = h->b.err;
        delete h;
        return st;
    }
    *out = h;
    return CGFDM_OK;
}

int cgfdm_batch_run(cgfdm_batch *b, int nsteps)
{
    if (!b) return CGFDM_E_ARG;
    return b->b.run(nsteps);
}

int cgfdm_batch_run_timed(cgfdm_batch *b, int nsteps, float *ms)
{
    if (!b || !ms) return CGFDM_E_ARG;
    return b->b.run(nsteps, ms);
}

int cgfdm_batch_destroy(cgfdm_batch *b)
{
    delete b;
    return CGFDM_OK;
}

const char *cgfdm_batch_last_error(const cgfdm_batch *b) { return b ? b->b.err.c_str() : g_create_error.c_str(); }

int cgfdm_destroy(cgfdm_session *s)
{
    delete s;
    return CGFDM_OK;
}

const char *cgfdm_last_error(const cgfdm_session *s)
{
    if (!s) return g_create_error.c_str();
    return s->s.err.c_str();
}

}  // extern "C"
