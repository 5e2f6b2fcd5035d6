/* fdtd_oracle_impl.h -- TEST INFRASTRUCTURE ONLY.  Body of the oracle time loop,
 * included twice by fdtd_oracle.c with REAL = double (suffix _f64) and REAL = float
 * (suffix _f32).  Every loop below restates one reference routine; citations are to
 * XiaofengYuChina/3D_FDTD_version008. */
#define O_CAT2(a, b) a##b
#define O_CAT(a, b) O_CAT2(a, b)
#define FN(name) O_CAT(name, SUFFIX)

static void *FN(o_alloc)(size_t n) {
    void *p = calloc(n ? n : 1, sizeof(REAL));
    return p;
}

static int64_t FN(oracle_run)(const oracle_case *c, oracle_state *s, uint64_t n0, uint64_t nsteps,
                              double *probe_out, int threads) {
    const size_t NxT = c->NxT, NyT = c->NyT, NzT = c->NzT, N = NxT * NyT * NzT;
    const size_t sI = NyT * NzT, sJ = NzT, sK = 1;
    const int npml = c->npml;
    const int gain = c->n_regions > 0 && c->region_map != NULL;
    const double dt = c->dt;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
    REAL *E[3], *H[3], *J[3], *bE[3], *psi[12];
    for (int q = 0; q < 3; ++q) {
        E[q] = FN(o_alloc)(N); H[q] = FN(o_alloc)(N); J[q] = FN(o_alloc)(N); bE[q] = FN(o_alloc)(N);
        for (size_t id = 0; id < N; ++id) {
            E[q][id] = (REAL)s->E[q][id];
            H[q][id] = (REAL)s->H[q][id];
            bE[q][id] = (REAL)c->bE[q][id];
        }
    }
    for (int q = 0; q < 12; ++q) psi[q] = FN(o_alloc)(N);
    /* psi order: Ex_y Ex_z Ey_z Ey_x Ez_x Ez_y | Hx_y Hx_z Hy_z Hy_x Hz_x Hz_y (src/boundary.hpp:92-97) */
    REAL *idx = FN(o_alloc)(NxT), *idy = FN(o_alloc)(NyT), *idz = FN(o_alloc)(NzT);
    REAL *rdx = FN(o_alloc)(NxT), *rdy = FN(o_alloc)(NyT), *rdz = FN(o_alloc)(NzT);
    for (size_t q = 0; q < NxT; ++q) { idx[q] = (REAL)c->inv_dx[q]; rdx[q] = (REAL)(1.0 / c->dx[q]); }
    for (size_t q = 0; q < NyT; ++q) { idy[q] = (REAL)c->inv_dy[q]; rdy[q] = (REAL)(1.0 / c->dy[q]); }
    for (size_t q = 0; q < NzT; ++q) { idz[q] = (REAL)c->inv_dz[q]; rdz[q] = (REAL)(1.0 / c->dz[q]); }
    const size_t Ns[3] = {NxT, NyT, NzT};
    REAL *kap[3], *bEp[3], *cEp[3], *bHp[3], *cHp[3];
    for (int a = 0; a < 3; ++a) {
        kap[a] = FN(o_alloc)(Ns[a]); bEp[a] = FN(o_alloc)(Ns[a]); cEp[a] = FN(o_alloc)(Ns[a]);
        bHp[a] = FN(o_alloc)(Ns[a]); cHp[a] = FN(o_alloc)(Ns[a]);
        for (size_t q = 0; q < Ns[a]; ++q) {
            kap[a][q] = (REAL)c->kappa[a][q];
            bEp[a][q] = (REAL)c->bEp[a][q]; cEp[a][q] = (REAL)c->cEp[a][q];
            bHp[a][q] = (REAL)c->bHp[a][q]; cHp[a][q] = (REAL)c->cHp[a][q];
        }
    }
    const REAL bH = (REAL)c->bH;
    REAL *Pz = NULL, *Pp = NULL, *dPdt = NULL, *Ezo = NULL, *Nu = NULL, *Ng = NULL, *Nd = NULL;
    if (gain) {
        Pz = FN(o_alloc)(N); Pp = FN(o_alloc)(N); dPdt = FN(o_alloc)(N); Ezo = FN(o_alloc)(N);
        Nu = FN(o_alloc)(N); Ng = FN(o_alloc)(N); Nd = FN(o_alloc)(N);
        for (size_t id = 0; id < N; ++id) {
            Pz[id] = (REAL)s->Pz[id]; Pp[id] = (REAL)s->Pz_prev[id];
            Nu[id] = (REAL)s->Nu[id]; Ng[id] = (REAL)s->Ng[id];
            const int r = c->region_map[id];
            Nd[id] = r >= 0 ? (REAL)c->regions[r].N0 : (REAL)0;
        }
    }
#define IN_PML(n, NT) ((((int)(n)) < ((int)(NT)) - 1 - ((int)(n)) ? ((int)(n)) : ((int)(NT)) - 1 - ((int)(n))) < npml)
    int64_t samples = 0;
    const int nprobe = c->n_probes;
    for (uint64_t n = n0; n < n0 + nsteps; ++n) {
        /* J reset + DipoleSource::inject_half_step (src/3D_FDTD_version008.cpp:270-275,
         * src/sources/dipole_source.hpp:60-85) */
        for (int q = 0; q < 3; ++q) memset(J[q], 0, N * sizeof(REAL));
        for (int q = 0; q < c->n_src; ++q) {
            const oracle_source *sr = &c->src[q];
            const double t_half = ((double)n + 0.5) * dt;
            const double Jval = waveform_value(sr->waveform, t_half, sr->I0, sr->f0, sr->tau, sr->t0, sr->t_shift) /
                                sr->cell_area;
            J[sr->comp][IDX3(sr->i, sr->j, sr->k, NyT, NzT)] += (REAL)Jval;
        }
        /* PlaneWaveSource::inject_half_step (src/sources/plane_wave_source.hpp:77-176),
         * registered after the dipoles */
        for (int q = 0; q < c->n_sheets; ++q) {
            const oracle_sheet *w = &c->sheets[q];
            const double t_half = ((double)n + 0.5) * dt;
            const double Et = waveform_value(w->waveform, t_half, w->E0, w->f0, w->tau, w->t0, w->t_shift);
            const double Jamp = 2.0 * Et / (376.730313668 * w->d) * w->sign;
            for (uint64_t a = w->lo0; a <= w->hi0; ++a)
                for (uint64_t b = w->lo1; b <= w->hi1; ++b) {
                    const uint64_t i = w->axis == 0 ? w->plane : a;
                    const uint64_t j = w->axis == 1 ? w->plane : w->axis == 0 ? a : b;
                    const uint64_t k = w->axis == 2 ? w->plane : b;
                    J[w->comp][IDX3(i, j, k, NyT, NzT)] += (REAL)Jamp;
                }
        }
        /* update_polarization_multi_region (src/two_level_system.hpp:574-609) */
        if (gain) {
#pragma omp parallel for
            for (long long id = 0; id < (long long)N; ++id) {
                if (Nd[id] <= 0) continue;
                const int r = c->region_map[id];
                if (r < 0) continue;
                const oracle_region *g = &c->regions[r];
                const REAL Ng_frac = (Nd[id] > 0) ? (Ng[id] - Nu[id]) / Nd[id] : (REAL)0;
#if ORACLE_IS_F64
                const REAL driving = Nd[id] * Ng_frac * E[2][id];
                const REAL Pn = g->kapa_coeff * driving + g->pa2 * Pz[id] + g->pa3 * Pp[id];
#else
                const REAL Pn = (REAL)(g->kapa_coeff * g->N0) * (Ng_frac * E[2][id]) + (REAL)g->pa2 * Pz[id] +
                                (REAL)g->pa3 * Pp[id];
#endif
                const REAL Po = Pz[id];
                Pp[id] = Po;
                Pz[id] = Pn;
                dPdt[id] = (Pn - Po) * (REAL)g->inv_dt;
            }
        }
        /* fdtd_update_H (src/fdtd_stepper.hpp:8-47), aH = 1 */
#pragma omp parallel for
        for (long long i = 0; i < (long long)NxT - 1; ++i)
            for (size_t j = 0; j < NyT - 1; ++j)
                for (size_t k = 0; k < NzT - 1; ++k) {
                    const size_t id = IDX3(i, j, k, NyT, NzT);
                    const REAL cx = (E[2][id + sJ] - E[2][id]) * idy[j] - (E[1][id + sK] - E[1][id]) * idz[k];
                    const REAL cy = (E[0][id + sK] - E[0][id]) * idz[k] - (E[2][id + sI] - E[2][id]) * idx[i];
                    const REAL cz = (E[1][id + sI] - E[1][id]) * idx[i] - (E[0][id + sJ] - E[0][id]) * idy[j];
                    H[0][id] = H[0][id] - bH * cx;
                    H[1][id] = H[1][id] - bH * cy;
                    H[2][id] = H[2][id] - bH * cz;
                }
        /* CPMLBoundary::apply_after_H (src/boundary.hpp:150-225) */
        if (npml > 0) {
#pragma omp parallel for
            for (long long i = 0; i < (long long)NxT - 1; ++i)
                for (size_t j = 0; j < NyT - 1; ++j)
                    for (size_t k = 0; k < NzT - 1; ++k) {
                        const size_t id = IDX3(i, j, k, NyT, NzT);
                        const REAL ix = rdx[i], iy = rdy[j], iz = rdz[k];
                        if (IN_PML(j, NyT)) {
                            REAL d = (E[2][id + sJ] - E[2][id]) * iy, corr = d / kap[1][j];
                            REAL *p = &psi[6][id]; *p = bHp[1][j] * *p + cHp[1][j] * d; corr += *p;
                            H[0][id] -= bH * (corr - d);
                        }
                        if (IN_PML(k, NzT)) {
                            REAL d = (E[1][id + sK] - E[1][id]) * iz, corr = d / kap[2][k];
                            REAL *p = &psi[7][id]; *p = bHp[2][k] * *p + cHp[2][k] * d; corr += *p;
                            H[0][id] -= bH * (-(corr - d));
                        }
                        if (IN_PML(k, NzT)) {
                            REAL d = (E[0][id + sK] - E[0][id]) * iz, corr = d / kap[2][k];
                            REAL *p = &psi[8][id]; *p = bHp[2][k] * *p + cHp[2][k] * d; corr += *p;
                            H[1][id] -= bH * (corr - d);
                        }
                        if (IN_PML(i, NxT)) {
                            REAL d = (E[2][id + sI] - E[2][id]) * ix, corr = d / kap[0][i];
                            REAL *p = &psi[9][id]; *p = bHp[0][i] * *p + cHp[0][i] * d; corr += *p;
                            H[1][id] -= bH * (-(corr - d));
                        }
                        if (IN_PML(i, NxT)) {
                            REAL d = (E[1][id + sI] - E[1][id]) * ix, corr = d / kap[0][i];
                            REAL *p = &psi[10][id]; *p = bHp[0][i] * *p + cHp[0][i] * d; corr += *p;
                            H[2][id] -= bH * (corr - d);
                        }
                        if (IN_PML(j, NyT)) {
                            REAL d = (E[0][id + sJ] - E[0][id]) * iy, corr = d / kap[1][j];
                            REAL *p = &psi[11][id]; *p = bHp[1][j] * *p + cHp[1][j] * d; corr += *p;
                            H[2][id] -= bH * (-(corr - d));
                        }
                    }
        }
        /* fdtd_update_E (src/fdtd_stepper.hpp:49-89) / fdtd_update_E_with_gain
         * (src/two_level_system.hpp:299-342), aE = 1 */
#pragma omp parallel for
        for (long long i = 1; i < (long long)NxT; ++i)
            for (size_t j = 1; j < NyT; ++j)
                for (size_t k = 1; k < NzT; ++k) {
                    const size_t id = IDX3(i, j, k, NyT, NzT);
                    const REAL cx = (H[2][id] - H[2][id - sJ]) * idy[j] - (H[1][id] - H[1][id - sK]) * idz[k];
                    const REAL cy = (H[0][id] - H[0][id - sK]) * idz[k] - (H[2][id] - H[2][id - sI]) * idx[i];
                    const REAL cz = (H[1][id] - H[1][id - sI]) * idx[i] - (H[0][id] - H[0][id - sJ]) * idy[j];
                    E[0][id] = E[0][id] + bE[0][id] * (cx - J[0][id]);
                    E[1][id] = E[1][id] + bE[1][id] * (cy - J[1][id]);
                    if (gain) {
                        Ezo[id] = E[2][id];
                        E[2][id] = E[2][id] + bE[2][id] * (cz - J[2][id] - dPdt[id]);
                    } else {
                        E[2][id] = E[2][id] + bE[2][id] * (cz - J[2][id]);
                    }
                }
        /* CPMLBoundary::apply_after_E (src/boundary.hpp:227-300) */
        if (npml > 0) {
#pragma omp parallel for
            for (long long i = 1; i < (long long)NxT; ++i)
                for (size_t j = 1; j < NyT; ++j)
                    for (size_t k = 1; k < NzT; ++k) {
                        const size_t id = IDX3(i, j, k, NyT, NzT);
                        const REAL ix = rdx[i], iy = rdy[j], iz = rdz[k];
                        if (IN_PML(j, NyT)) {
                            REAL d = (H[2][id] - H[2][id - sJ]) * iy, corr = d / kap[1][j];
                            REAL *p = &psi[0][id]; *p = bEp[1][j] * *p + cEp[1][j] * d; corr += *p;
                            E[0][id] += bE[0][id] * (corr - d);
                        }
                        if (IN_PML(k, NzT)) {
                            REAL d = (H[1][id] - H[1][id - sK]) * iz, corr = d / kap[2][k];
                            REAL *p = &psi[1][id]; *p = bEp[2][k] * *p + cEp[2][k] * d; corr += *p;
                            E[0][id] += bE[0][id] * (-(corr - d));
                        }
                        if (IN_PML(k, NzT)) {
                            REAL d = (H[0][id] - H[0][id - sK]) * iz, corr = d / kap[2][k];
                            REAL *p = &psi[2][id]; *p = bEp[2][k] * *p + cEp[2][k] * d; corr += *p;
                            E[1][id] += bE[1][id] * (corr - d);
                        }
                        if (IN_PML(i, NxT)) {
                            REAL d = (H[2][id] - H[2][id - sI]) * ix, corr = d / kap[0][i];
                            REAL *p = &psi[3][id]; *p = bEp[0][i] * *p + cEp[0][i] * d; corr += *p;
                            E[1][id] += bE[1][id] * (-(corr - d));
                        }
                        if (IN_PML(i, NxT)) {
                            REAL d = (H[1][id] - H[1][id - sI]) * ix, corr = d / kap[0][i];
                            REAL *p = &psi[4][id]; *p = bEp[0][i] * *p + cEp[0][i] * d; corr += *p;
                            E[2][id] += bE[2][id] * (corr - d);
                        }
                        if (IN_PML(j, NyT)) {
                            REAL d = (H[0][id] - H[0][id - sJ]) * iy, corr = d / kap[1][j];
                            REAL *p = &psi[5][id]; *p = bEp[1][j] * *p + cEp[1][j] * d; corr += *p;
                            E[2][id] += bE[2][id] * (-(corr - d));
                        }
                    }
        }
        /* PECBoundary::apply_after_E (src/boundary.hpp:55-74): E = 0 on the six faces */
        if (c->pec) {
            for (size_t j = 0; j < NyT; ++j)
                for (size_t k = 0; k < NzT; ++k)
                    for (int q = 0; q < 3; ++q) E[q][IDX3(0, j, k, NyT, NzT)] = E[q][IDX3(NxT - 1, j, k, NyT, NzT)] = 0;
            for (size_t i = 0; i < NxT; ++i)
                for (size_t k = 0; k < NzT; ++k)
                    for (int q = 0; q < 3; ++q) E[q][IDX3(i, 0, k, NyT, NzT)] = E[q][IDX3(i, NyT - 1, k, NyT, NzT)] = 0;
            for (size_t i = 0; i < NxT; ++i)
                for (size_t j = 0; j < NyT; ++j)
                    for (int q = 0; q < 3; ++q) E[q][IDX3(i, j, 0, NyT, NzT)] = E[q][IDX3(i, j, NzT - 1, NyT, NzT)] = 0;
        }
        /* PointFieldDetector::record_after_E (src/detectors/point_field_detector.hpp:242-255) */
        if (n % c->save_every == 0) {
            if (probe_out)
                for (int q = 0; q < nprobe; ++q)
                    probe_out[(size_t)samples * nprobe + q] =
                        PROBE_VALUE(REAL, c->probe_comp[q], (size_t)c->probe_idx[q], E, H);
            ++samples;
        }
        /* update_populations_multi_region (src/two_level_system.hpp:612-666); the pump term
         * is this library's extension (absent from the reference, 0 reproduces it). */
        if (gain) {
#pragma omp parallel for
            for (long long id = 0; id < (long long)N; ++id) {
                if (Nd[id] <= 0) continue;
                const int r = c->region_map[id];
                if (r < 0) continue;
                const oracle_region *g = &c->regions[r];
                const REAL Nu_curr = Nu[id];
                const REAL Ntotal = Nd[id];
                if (Ntotal <= 0) continue;
                const REAL inv_tau = (REAL)(1.0 / g->tau);
                const REAL inv_hbar_omega = (REAL)(1.0 / (g->hbar * g->omega_a));
                const REAL E_avg = (REAL)0.5 * (E[2][id] + Ezo[id]);
                const REAL delta_P = Pz[id] - Pp[id];
                const REAL stim = E_avg * delta_P * (REAL)g->inv_dt * inv_hbar_omega;
                REAL dNu = -inv_tau * Nu_curr + stim;
                REAL dNg = +inv_tau * Nu_curr - stim;
                if (g->pump_rate != 0.0) {
                    dNu += (REAL)g->pump_rate * Ng[id];
                    dNg -= (REAL)g->pump_rate * Ng[id];
                }
                Nu[id] += (REAL)dt * dNu;
                Ng[id] += (REAL)dt * dNg;
                Nu[id] = Nu[id] > 0 ? Nu[id] : (REAL)0;
                Ng[id] = Ng[id] > 0 ? Ng[id] : (REAL)0;
                if (g->clamp) {
                    REAL total = Nu[id] + Ng[id];
                    if (total > (REAL)1e-30) {
                        REAL scale = Ntotal / total;
                        Nu[id] *= scale;
                        Ng[id] *= scale;
                    }
                    Nu[id] = Nu[id] < Ntotal ? Nu[id] : Ntotal;
                    Ng[id] = Ntotal - Nu[id];
                }
            }
        }
    }
#undef IN_PML
    for (int q = 0; q < 3; ++q)
        for (size_t id = 0; id < N; ++id) {
            s->E[q][id] = (double)E[q][id];
            s->H[q][id] = (double)H[q][id];
        }
    if (gain) {
        for (size_t id = 0; id < N; ++id) {
            s->Pz[id] = (double)Pz[id]; s->Pz_prev[id] = (double)Pp[id];
            s->Nu[id] = (double)Nu[id]; s->Ng[id] = (double)Ng[id];
        }
        free(Pz); free(Pp); free(dPdt); free(Ezo); free(Nu); free(Ng); free(Nd);
    }
    for (int q = 0; q < 3; ++q) { free(E[q]); free(H[q]); free(J[q]); free(bE[q]); }
    for (int q = 0; q < 12; ++q) free(psi[q]);
    free(idx); free(idy); free(idz); free(rdx); free(rdy); free(rdz);
    for (int a = 0; a < 3; ++a) { free(kap[a]); free(bEp[a]); free(cEp[a]); free(bHp[a]); free(cHp[a]); }
    return samples;
}

#undef FN
#undef O_CAT
#undef O_CAT2
