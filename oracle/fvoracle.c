/*
 * fvoracle.c — CPU restatement of fvhyper's explicit FV step (test
 * infrastructure only; see fvoracle.h).  Every function cites the reference
 * code it restates, relative to the reference repository root.
 */
#include "fvoracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static inline double dmin(double a, double b) { return (b < a) ? b : a; } /* std::min */
static inline double dmax(double a, double b) { return (a < b) ? b : a; } /* std::max */

/* ---------------------------------------------------------------- mesh -- */
typedef struct { uint64_t* key; int64_t* val; uint64_t mask; } edge_map;

static uint64_t mix64(uint64_t x) {
    x ^= x >> 33; x *= 0xff51afd7ed558ccdULL; x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ULL; x ^= x >> 33;
    return x;
}
static int64_t* em_slot(edge_map* m, uint64_t k, int* found) {
    uint64_t h = mix64(k) & m->mask;
    while (m->key[h] != UINT64_MAX) {
        if (m->key[h] == k) { *found = 1; return &m->val[h]; }
        h = (h + 1) & m->mask;
    }
    *found = 0;
    m->key[h] = k;
    return &m->val[h];
}
static uint64_t ekey(uint32_t a, uint32_t b) {
    uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
    return ((uint64_t)lo << 32) | hi;
}

/* mesh::read_file after parsing (mesh.cpp:821-853): add_cell_edges
 * (mesh.cpp:130-154), convert_node_face_info (157-187), compute_mesh
 * (190-260), add_boundary_cells (623-669). */
int fvo_mesh_build(int64_t n_nodes, const double* X, const double* Y, int64_t nc,
                   const int32_t* cells4, int64_t nb, const int32_t* bnd_nodes,
                   const int32_t* bnd_group, fvo_mesh* o) {
    memset(o, 0, sizeof(*o));
    uint64_t cap = 16;
    while (cap < (uint64_t)(4 * nc + 16)) cap <<= 1;
    edge_map em = {malloc(cap * 8), malloc(cap * 8), cap - 1};
    memset(em.key, 0xff, cap * 8);
    int64_t emax = 4 * nc + 4;
    uint32_t* ec = malloc(emax * 2 * sizeof(uint32_t));
    uint32_t* en = malloc(emax * 2 * sizeof(uint32_t));
    int64_t E = 0;
    for (int64_t c = 0; c < nc; ++c) {
        const int32_t* cn = cells4 + 4 * c;
        int sz = cn[3] < 0 ? 3 : 4;
        for (int i = 0; i < sz; ++i) {
            int j = (i < sz - 1) ? i + 1 : 0;
            int found;
            int64_t* v = em_slot(&em, ekey(cn[i], cn[j]), &found);
            if (!found) {
                *v = E;
                ec[2 * E] = (uint32_t)c; ec[2 * E + 1] = 0;
                en[2 * E] = cn[i]; en[2 * E + 1] = cn[j];
                ++E;
            }
        }
    }
    for (int64_t c = 0; c < nc; ++c) { /* convert_node_face_info */
        const int32_t* cn = cells4 + 4 * c;
        int sz = cn[3] < 0 ? 3 : 4;
        for (int i = 0; i < sz; ++i) {
            int j = (i < sz - 1) ? i + 1 : 0;
            int found;
            int64_t e = *em_slot(&em, ekey(cn[i], cn[j]), &found);
            if ((uint32_t)c != ec[2 * e]) ec[2 * e + 1] = (uint32_t)c;
        }
    }
    int64_t nt = nc + nb;
    o->n_nodes = n_nodes; o->n_real = nc; o->n_total = nt; o->n_edges = E; o->n_bound = nb;
    o->edge_cells = ec; o->edge_nodes = en;
    o->enx = malloc(E * 8); o->eny = malloc(E * 8); o->elen = malloc(E * 8);
    o->ecx = malloc(E * 8); o->ecy = malloc(E * 8);
    o->area = malloc(nt * 8); o->ccx = malloc(nt * 8); o->ccy = malloc(nt * 8);
    o->bound_edges = malloc((nb + 1) * 4); o->bound_group = malloc((nb + 1) * 4);
    for (int64_t c = 0; c < nc; ++c) { /* centroids, mesh.cpp:194-206 */
        const int32_t* cn = cells4 + 4 * c;
        int sz = cn[3] < 0 ? 3 : 4;
        double cx = 0., cy = 0.;
        for (int j = 0; j < sz; ++j) {
            cx += X[cn[j]] / ((double)sz);
            cy += Y[cn[j]] / ((double)sz);
        }
        o->ccx[c] = cx; o->ccy[c] = cy;
    }
    for (int64_t e = 0; e < E; ++e) { /* edge centres and normals, mesh.cpp:210-229 */
        uint32_t a = en[2 * e], b = en[2 * e + 1];
        o->ecx[e] = (X[b] + X[a]) * 0.5;
        o->ecy[e] = (Y[b] + Y[a]) * 0.5;
        double dex = X[b] - X[a], dey = Y[b] - Y[a];
        double l = sqrt(dex * dex + dey * dey);
        o->elen[e] = l;
        o->enx[e] = -dey / l;
        o->eny[e] = dex / l;
        uint32_t c0 = ec[2 * e];
        double dot = o->enx[e] * (o->ecx[e] - o->ccx[c0]) + o->eny[e] * (o->ecy[e] - o->ccy[c0]);
        if (dot < 0) { o->enx[e] *= -1.; o->eny[e] *= -1.; }
    }
    for (int64_t c = 0; c < nc; ++c) { /* areas, mesh.cpp:232-259 */
        const int32_t* cn = cells4 + 4 * c;
        double x1 = X[cn[0]], x2 = X[cn[1]], x3 = X[cn[2]];
        double y1 = Y[cn[0]], y2 = Y[cn[1]], y3 = Y[cn[2]];
        if (cn[3] < 0) {
            o->area[c] = 0.5 * fabs(x1 * (y2 - y3) + x2 * (y3 - y1) + x3 * (y1 - y2));
        } else {
            double x4 = X[cn[3]], y4 = Y[cn[3]];
            o->area[c] = 0.5 * fabs(x1 * (y2 - y3) + x2 * (y3 - y1) + x3 * (y1 - y2)) +
                         0.5 * fabs(x1 * (y3 - y4) + x3 * (y4 - y1) + x4 * (y1 - y3));
        }
    }
    for (int64_t b = 0; b < nb; ++b) { /* ghost cells, mesh.cpp:623-669 */
        int found;
        int64_t* v = em_slot(&em, ekey(bnd_nodes[2 * b], bnd_nodes[2 * b + 1]), &found);
        if (!found) { free(em.key); free(em.val); fvo_mesh_free(o); return -1; }
        int64_t e = *v;
        uint32_t cell = ec[2 * e];
        double dx = o->ecx[e] - o->ccx[cell], dy = o->ecy[e] - o->ccy[cell];
        double dist = sqrt(dx * dx + dy * dy);
        int64_t g = nc + b;
        o->area[g] = o->area[cell];
        o->ccx[g] = o->ecx[e] + dist * o->enx[e];
        o->ccy[g] = o->ecy[e] + dist * o->eny[e];
        ec[2 * e + 1] = (uint32_t)g;
        o->bound_edges[b] = (uint32_t)e;
        o->bound_group[b] = bnd_group[b];
    }
    free(em.key); free(em.val);
    return 0;
}

void fvo_mesh_free(fvo_mesh* m) {
    free(m->edge_cells); free(m->edge_nodes); free(m->enx); free(m->eny); free(m->elen);
    free(m->ecx); free(m->ecy); free(m->area); free(m->ccx); free(m->ccy);
    free(m->bound_edges); free(m->bound_group);
    memset(m, 0, sizeof(*m));
}

/* ------------------------------------------------------------- physics -- */
static inline double pres(double gm1, const double* q) { /* calc_p, forwardStep/main.cpp:37-39 */
    return gm1 * (q[3] - 0.5 / q[0] * (q[1] * q[1] + q[2] * q[2]));
}

/* Roe flux with the "cures" eigenvalues.  ROE_FS follows
 * examples/forwardStep/main.cpp:72-135 (central part summed as one
 * expression); ROE_ST follows examples/shockTube/main.cpp:68-135 and
 * examples/naca/main.cpp:71-137 (central part accumulated side by side).  The
 * two differ only in the association of the central-flux sums. */
static void roe(double gamma, int fs_assoc, double* f, const double* qi, const double* qj,
                const double* n) {
    double pi = (gamma - 1) * (qi[3] - 0.5 / qi[0] * (qi[1] * qi[1] + qi[2] * qi[2]));
    double pj = (gamma - 1) * (qj[3] - 0.5 / qj[0] * (qj[1] * qj[1] + qj[2] * qj[2]));
    double Vi = (qi[1] * n[0] + qi[2] * n[1]) / qi[0];
    double Vj = (qj[1] * n[0] + qj[2] * n[1]) / qj[0];
    if (fs_assoc) {
        f[0] = (qi[0] * Vi + qj[0] * Vj) * 0.5;
        f[1] = (qi[1] * Vi + pi * n[0] + qj[1] * Vj + pj * n[0]) * 0.5;
        f[2] = (qi[2] * Vi + pi * n[1] + qj[2] * Vj + pj * n[1]) * 0.5;
        f[3] = ((qi[3] + pi) * Vi + (qj[3] + pj) * Vj) * 0.5;
    } else {
        f[0] = qi[0] * Vi;
        f[1] = qi[1] * Vi + pi * n[0];
        f[2] = qi[2] * Vi + pi * n[1];
        f[3] = (qi[3] + pi) * Vi;
        f[0] += qj[0] * Vj;
        f[1] += qj[1] * Vj + pj * n[0];
        f[2] += qj[2] * Vj + pj * n[1];
        f[3] += (qj[3] + pj) * Vj;
        for (int i = 0; i < 4; ++i) f[i] *= 0.5;
    }
    const double pL = pi, pR = pj;
    const double uL = qi[1] / qi[0], vL = qi[2] / qi[0];
    const double uR = qj[1] / qj[0], vR = qj[2] / qj[0];
    const double srhoL = sqrt(qi[0]), srhoR = sqrt(qj[0]);
    const double rho = srhoR * srhoL;
    const double u = (uL * srhoL + uR * srhoR) / (srhoL + srhoR);
    const double v = (vL * srhoL + vR * srhoR) / (srhoL + srhoR);
    const double h = ((qi[3] + pL) / qi[0] * srhoL + (qj[3] + pR) / qj[0] * srhoR) / (srhoL + srhoR);
    const double q2 = u * u + v * v;
    const double c = sqrt((gamma - 1.) * (h - 0.5 * q2));
    const double V = u * n[0] + v * n[1];
    const double VR = uR * n[0] + vR * n[1];
    const double VL = uL * n[0] + vL * n[1];
    const double lambda_cm = fabs(dmin(V - c, VL - c));
    const double lambda_c = fabs(V);
    const double lambda_cp = fabs(dmax(V + c, VR + c));
    const double kF1 = lambda_cm * ((pR - pL) - rho * c * (VR - VL)) / (2. * c * c);
    const double kF234_0 = lambda_c * ((qj[0] - qi[0]) - (pR - pL) / (c * c));
    const double kF234_1 = lambda_c * rho;
    const double kF5 = lambda_cp * ((pR - pL) + rho * c * (VR - VL)) / (2. * c * c);
    f[0] -= 0.5 * (kF1 + kF234_0 + kF5);
    f[1] -= 0.5 * (kF1 * (u - c * n[0]) + kF234_0 * u + kF234_1 * (uR - uL - (VR - VL) * n[0]) + kF5 * (u + c * n[0]));
    f[2] -= 0.5 * (kF1 * (v - c * n[1]) + kF234_0 * v + kF234_1 * (vR - vL - (VR - VL) * n[1]) + kF5 * (v + c * n[1]));
    f[3] -= 0.5 * (kF1 * (h - c * V) + kF234_0 * q2 * 0.5 + kF234_1 * (u * (uR - uL) + v * (vR - vL) - V * (VR - VL)) + kF5 * (h + c * V));
}

/* Upwind advection flux, examples/burgers/main.cpp:68-96 (V = 2). */
static void burgers(double* f, const double* qi, const double* qj, const double* n) {
    double Vi = qi[0] * n[0] + qi[1] * n[1];
    double Vj = qj[0] * n[0] + qj[1] * n[1];
    double fi0 = Vi * qi[0], fi1 = Vi * qi[1];
    double fj0 = Vj * qj[0], fj1 = Vj * qj[1];
    double V = dmax(fabs(Vi), fabs(Vj));
    f[0] = 0.5 * (fi0 + fj0) - 0.5 * V * (qj[0] - qi[0]);
    f[1] = 0.5 * (fi1 + fj1) - 0.5 * V * (qj[1] - qi[1]);
}

void fvo_flux(const fvo_physics* ph, double* f, const double* qi, const double* qj, const double* n) {
    if (ph->flux == FVO_FLUX_BURGERS) burgers(f, qi, qj, n);
    else roe(ph->gamma, ph->flux == FVO_FLUX_ROE_FS, f, qi, qj, n);
}

static void ns_viscous(const fvo_physics* ph, double* f, const double* qi, const double* qj,
                       const double* gx, const double* gy, const double* n);

/* calc_flux with the face gradient it receives (explicit.cpp:342): the
 * diffusion and Navier-Stokes kinds read it, the others ignore it. */
void fvo_flux_grad(const fvo_physics* ph, double* f, const double* qi, const double* qj, const double* gx,
                   const double* gy, const double* n) {
    if (ph->flux == FVO_FLUX_DIFFUSION) {
        f[0] = -(gx[0] * n[0] + gy[0] * n[1]);
    } else if (ph->flux == FVO_FLUX_BURGERS_DIFF) {  /* tests/tests.cpp:94-116 */
        burgers(f, qi, qj, n);
        f[0] += -(gx[0] * n[0] + gy[0] * n[1]);
        f[1] += -(gx[1] * n[0] + gy[1] * n[1]);
    } else if (ph->flux == FVO_FLUX_NS) {
        roe(ph->gamma, 0, f, qi, qj, n);
        ns_viscous(ph, f, qi, qj, gx, gy, n);
    } else {
        fvo_flux(ph, f, qi, qj, n);
    }
}

/* Viscous part of the Navier-Stokes flux, examples/flatPlate/main.cpp:193-224
 * (= nacaTransient/main.cpp:197-228) with its helpers calc_p, calc_grad_p,
 * calc_grad_t, calc_grad_u, calc_grad_v (flatPlate/main.cpp:38-92): stresses
 * and heat flux at the mean of the two face states, from the face gradient
 * (gx, gy); subtracted from the Roe flux f. */
static void ns_viscous(const fvo_physics* ph, double* f, const double* qi, const double* qj,
                       const double* gx, const double* gy, const double* n) {
    const double gamma = ph->gamma, mu = ph->mu;
    double q[4];
    for (int i = 0; i < 4; ++i) q[i] = 0.5 * (qi[i] + qj[i]);
    const double p = (gamma - 1) * (q[3] - 0.5 / q[0] * (q[1] * q[1] + q[2] * q[2]));
    double gp0 = 2. * gx[3];
    gp0 -= gx[1] * q[1] / q[0] + q[1] * (gx[1] * q[0] - gx[0] * q[1]) / (q[0] * q[0]);
    gp0 -= gx[2] * q[2] / q[0] + q[2] * (gx[2] * q[0] - gx[0] * q[2]) / (q[0] * q[0]);
    gp0 *= 0.5 * (gamma - 1);
    double gp1 = 2. * gy[3];
    gp1 -= gy[1] * q[1] / q[0] + q[1] * (gy[1] * q[0] - gy[0] * q[1]) / (q[0] * q[0]);
    gp1 -= gy[2] * q[2] / q[0] + q[2] * (gy[2] * q[0] - gy[0] * q[2]) / (q[0] * q[0]);
    gp1 *= 0.5 * (gamma - 1);
    const double gt0 = (1. / ph->r) * ((gp0 * q[0] - gx[0] * p) / (q[0] * q[0]));
    const double gt1 = (1. / ph->r) * ((gp1 * q[0] - gy[0] * p) / (q[0] * q[0]));
    const double gu0 = (q[0] * gx[1] - q[1] * gx[0]) / (q[0] * q[0]);
    const double gu1 = (q[0] * gy[1] - q[1] * gy[0]) / (q[0] * q[0]);
    const double gv0 = (q[0] * gx[2] - q[2] * gx[0]) / (q[0] * q[0]);
    const double gv1 = (q[0] * gy[2] - q[2] * gy[0]) / (q[0] * q[0]);
    const double div_v = gu0 + gv1;
    const double tau_xx = 2. * mu * (gu0 - div_v / 3.);
    const double tau_yy = 2. * mu * (gv1 - div_v / 3.);
    const double tau_xy = mu * (gu1 + gv0);
    const double k = ph->cp * mu / ph->pr;
    const double phi0 = q[1] / q[0] * tau_xx + q[2] / q[0] * tau_xy + k * gt0;
    const double phi1 = q[1] / q[0] * tau_xy + q[2] / q[0] * tau_yy + k * gt1;
    f[1] -= n[0] * tau_xx + n[1] * tau_xy;
    f[2] -= n[0] * tau_xy + n[1] * tau_yy;
    f[3] -= n[0] * phi0 + n[1] * phi1;
}

/* Boundary conditions.  COPY: examples/shockTube/main.cpp:158-163.  WALL:
 * examples/forwardStep/main.cpp:262-269.  INLET_OUTLET:
 * examples/forwardStep/main.cpp:194-261.  FARFIELD: examples/naca/main.cpp:
 * 192-259.  The subsonic outlet branches keep the reference's
 * b[2] = b[1]*(...) (forwardStep/main.cpp:257, naca/main.cpp:255).
 * NOSLIP: examples/flatPlate/main.cpp:361-366.  FARFIELD_B0:
 * examples/flatPlate/main.cpp:286-352 (= nacaTransient/main.cpp:294-360),
 * FARFIELD with b[2] = b[0]*(...) in both subsonic branches. */
static void bc_state(const fvo_physics* ph, int group, const double* bv, double* b, const double* q,
                     const double* n);

void fvo_bc(const fvo_physics* ph, int group, double* b, const double* q, const double* n) {
    bc_state(ph, group, ph->group_bv + 4 * group, b, q, n);
}

static void bc_state(const fvo_physics* ph, int group, const double* bv, double* b, const double* q,
                     const double* n) {
    const int kind = ph->group_bc[group];
    const double gamma = ph->gamma;
    const int V = ph->V;
    if (kind == FVO_BC_COPY) {
        for (int k = 0; k < V; ++k) b[k] = q[k];
        return;
    }
    if (kind == FVO_BC_WALL) {
        b[0] = q[0];
        b[1] = q[1] - 2.0 * n[0] * (n[0] * q[1] + n[1] * q[2]);
        b[2] = q[2] - 2.0 * n[1] * (n[0] * q[1] + n[1] * q[2]);
        b[3] = q[3];
        return;
    }
    if (kind == FVO_BC_TANGENT) {
        b[0] = -n[1];
        b[1] = n[0];
        return;
    }
    if (kind == FVO_BC_NOSLIP) {
        b[0] = q[0];
        b[1] = -q[1];
        b[2] = -q[2];
        b[3] = q[3];
        return;
    }
    const int b0 = kind == FVO_BC_FARFIELD_B0;  /* tangential momentum from b[0] */
    double U0 = q[1] / q[0], U1 = q[2] / q[0];
    double u_norm = sqrt(U0 * U0 + U1 * U1);
    double u_dot_n = U0 * n[0] + U1 * n[1];
    double p = (gamma - 1) * (q[3] - 0.5 / q[0] * (q[1] * q[1] + q[2] * q[2]));
    double c = sqrt(gamma * p / q[0]);
    double mach = u_norm / c;
    if (mach > 1) {
        if (u_dot_n < 0) { for (int k = 0; k < 4; ++k) b[k] = bv[k]; }
        else { for (int k = 0; k < 4; ++k) b[k] = q[k]; }
        return;
    }
    double pa = (gamma - 1) * (bv[3] - 0.5 / bv[0] * (bv[1] * bv[1] + bv[2] * bv[2]));
    double rhoa = bv[0], ua = bv[1] / bv[0], va = bv[2] / bv[0];
    double pd = p, rhod = q[0], ud = q[1] / q[0], vd = q[2] / q[0];
    double rho0 = q[0], c0 = c;
    if (u_dot_n < 0) {
        if (kind == FVO_BC_INLET_OUTLET) {
            double pb = pd;
            b[0] = bv[0]; b[1] = bv[1]; b[2] = bv[2];
            b[3] = pb / (gamma - 1.) + 0.5 / b[0] * (b[1] * b[1] + b[2] * b[2]);
        } else {
            double pb = 0.5 * (pa + pd - rho0 * c0 * (n[0] * (ua - ud) + n[1] * (va - vd)));
            b[0] = rhoa + (pb - pa) / (c0 * c0);
            b[1] = b[0] * (ua - n[0] * (pa - pb) / (rho0 * c0));
            b[2] = b[b0 ? 0 : 1] * (va - n[1] * (pa - pb) / (rho0 * c0));
            b[3] = pb / (gamma - 1) + 0.5 / b[0] * (b[1] * b[1] + b[2] * b[2]);
        }
    } else {
        double pb = pa;
        b[0] = rhod + (pb - pd) / (c0 * c0);
        b[1] = b[0] * (ud + n[0] * (pd - pb) / (rho0 * c0));
        b[2] = b[b0 ? 0 : 1] * (va + n[1] * (pd - pb) / (rho0 * c0));
        b[3] = pb / (gamma - 1.) + 0.5 / b[0] * (b[1] * b[1] + b[2] * b[2]);
    }
    (void)rhoa;
}

/* Limiter functions phi.  ZERO: examples/shockTube/main.cpp:60-62.
 * MICHALAK (y_t = 2): examples/forwardStep/main.cpp:57-66.  MINMOD:
 * examples/burgers/main.cpp:51-53.  VENKAT: phi(y) = (y^2+2y)/(y^2+y+2),
 * Venkatakrishnan, J. Comput. Phys. 118 (1995); not in the reference. */
double fvo_limiter_func(const fvo_physics* ph, double y) {
    switch (ph->limiter) {
    case FVO_LIM_MICHALAK: {
        const double yt = 2.0;
        if (y >= yt) return 1.0;
        const double a = 1.0 / (yt * yt) - 2.0 / (yt * yt * yt);
        const double b = -3.0 / 2.0 * a * yt - 0.5 / yt;
        return a * y * y * y + b * y * y + y;
    }
    case FVO_LIM_VENKAT: return (y * y + 2.0 * y) / (y * y + y + 2.0);
    case FVO_LIM_MINMOD: return dmax(0., dmin(1., y));
    default: return 0.;
    }
}

/* ------------------------------------------------------------ stages -- */
/* Viscous time steps (C = 2).  VISC_MIN: examples/flatPlate/main.cpp:230-277,
 * dt = min over faces of cfl A / (convective + C viscous eigenvalue), from 1.
 * VISC_SUM: examples/nacaTransient/main.cpp:234-285, dt = cfl A / sum over
 * faces of le * max of the two sides' (convective + C viscous) eigenvalues. */
static void calc_dt_viscous(const fvo_mesh* m, const fvo_physics* ph, const double* q, double* dt) {
    const double gamma = ph->gamma, gm1 = gamma - 1, cfl = ph->cfl, C = 2;
    const int sum = ph->dt_kind == FVO_DT_VISC_SUM;
    for (int64_t i = 0; i < m->n_total; ++i) dt[i] = sum ? 0. : 1.0;
    for (int64_t e = 0; e < m->n_edges; ++e) {
        uint32_t i = m->edge_cells[2 * e], j = m->edge_cells[2 * e + 1];
        double le = m->elen[e], n0 = m->enx[e], n1 = m->eny[e];
        const double* qi = q + 4 * (size_t)i;
        const double* qj = q + 4 * (size_t)j;
        double ci = sqrt(pres(gm1, qi) * gamma / qi[0]);
        double cj = sqrt(pres(gm1, qj) * gamma / qj[0]);
        double eig_vi = dmax(4. / (3. * qi[0]), gamma / qi[0]) * (ph->mu / ph->pr) * le * le / m->area[i];
        double eig_vj = dmax(4. / (3. * qj[0]), gamma / qj[0]) * (ph->mu / ph->pr) * le * le / m->area[j];
        if (sum) {
            double eig_ci = ci + fabs(qi[1] / qi[0] * n0 + qi[2] / qi[0] * n1);
            double eig_cj = cj + fabs(qj[1] / qj[0] * n0 + qj[2] / qj[0] * n1);
            double center = dmax(eig_ci + C * eig_vi, eig_cj + C * eig_vj);
            dt[i] += center * le;
            dt[j] += center * le;
        } else {
            double eig_ci = (ci + fabs(n0 * qi[1] / qi[0]) + fabs(n1 * qi[2] / qi[0])) * le;
            double eig_cj = (cj + fabs(n0 * qj[1] / qj[0]) + fabs(n1 * qj[2] / qj[0])) * le;
            double dti = cfl * m->area[i] / (eig_ci + C * eig_vi);
            double dtj = cfl * m->area[j] / (eig_cj + C * eig_vj);
            dt[i] = dmin(dt[i], dti);
            dt[j] = dmin(dt[j], dtj);
        }
    }
    if (sum)
        for (int64_t i = 0; i < m->n_total; ++i) dt[i] = cfl * m->area[i] / dt[i];
}

/* Time step kinds.  CFL_SUM: examples/forwardStep/main.cpp:140-185.
 * CFL_MIN_SIGNED: examples/naca/main.cpp:142-183.  CONST:
 * examples/shockTube/main.cpp:140-147.  dt is one value per cell (the
 * reference stores it V times per cell, all equal). */
void fvo_calc_dt(const fvo_mesh* m, const fvo_physics* ph, const double* q, double* dt) {
    const int V = ph->V;
    const double gamma = ph->gamma, gm1 = gamma - 1;
    if (ph->dt_kind == FVO_DT_CONST) {
        for (int64_t i = 0; i < m->n_total; ++i) dt[i] = ph->dt_const;
        return;
    }
    if (ph->dt_kind == FVO_DT_VISC_MIN || ph->dt_kind == FVO_DT_VISC_SUM) {
        calc_dt_viscous(m, ph, q, dt);
        return;
    }
    const int sum = ph->dt_kind == FVO_DT_CFL_SUM;
    for (int64_t i = 0; i < m->n_total; ++i) dt[i] = sum ? 0. : 1.0;
    for (int64_t e = 0; e < m->n_edges; ++e) {
        uint32_t i = m->edge_cells[2 * e], j = m->edge_cells[2 * e + 1];
        double le = m->elen[e], n0 = m->enx[e], n1 = m->eny[e];
        const double* qi = q + (size_t)V * i;
        const double* qj = q + (size_t)V * j;
        double ci = sqrt(pres(gm1, qi) * gamma / qi[0]);
        double cj = sqrt(pres(gm1, qj) * gamma / qj[0]);
        if (sum) {
            double ei = ci + fabs(qi[1] / qi[0] * n0 + qi[2] / qi[0] * n1);
            double ej = cj + fabs(qj[1] / qj[0] * n0 + qj[2] / qj[0] * n1);
            double center = dmax(ei, ej);
            dt[i] += center * le;
            dt[j] += center * le;
        } else {
            double ei = (ci + fabs(qi[1] / qi[0])) * n0 + (ci + fabs(qi[2] / qi[0])) * n1;
            double ej = (cj + fabs(qj[1] / qj[0])) * n0 + (cj + fabs(qj[2] / qj[0])) * n1;
            double dti = ph->cfl * (m->area[i] / le) / fabs(ei);
            double dtj = ph->cfl * (m->area[j] / le) / fabs(ej);
            dt[i] = dmin(dt[i], dti);
            dt[j] = dmin(dt[j], dtj);
        }
    }
    if (sum)
        for (int64_t i = 0; i < m->n_total; ++i) dt[i] = ph->cfl * m->area[i] / dt[i];
}

/* min_dt, explicit.cpp:555-564 (over every cell, boundary ghosts included). */
void fvo_min_dt(const fvo_mesh* m, double* dt) {
    double mn = dt[0];
    for (int64_t i = 0; i < m->n_total; ++i) mn = dmin(mn, dt[i]);
    for (int64_t i = 0; i < m->n_total; ++i) dt[i] = mn;
}

/* Green-Gauss gradients, explicit.cpp:112-171. */
void fvo_calc_gradients(const fvo_mesh* m, const fvo_physics* ph, const double* q, double* gx, double* gy) {
    const int V = ph->V;
    memset(gx, 0, sizeof(double) * V * m->n_total);
    memset(gy, 0, sizeof(double) * V * m->n_total);
    for (int64_t e = 0; e < m->n_edges; ++e) {
        uint32_t i = m->edge_cells[2 * e], j = m->edge_cells[2 * e + 1];
        double nx = m->enx[e], ny = m->eny[e], le = m->elen[e];
        double dxif = m->ecx[e] - m->ccx[i], dyif = m->ecy[e] - m->ccy[i];
        double dif = sqrt(dxif * dxif + dyif * dyif);
        double dxij = m->ccx[i] - m->ccx[j], dyij = m->ccy[i] - m->ccy[j];
        double dij = sqrt(dxij * dxij + dyij * dyij);
        double g = dif / dij;
        if (i != j) {
            for (int k = 0; k < V; ++k) {
                double f = (q[V * i + k] * (1.0 - g) + q[V * j + k] * g) * le;
                gx[V * i + k] += f * nx;
                gy[V * i + k] += f * ny;
                gx[V * j + k] -= f * nx;
                gy[V * j + k] -= f * ny;
            }
        }
    }
    for (int64_t i = 0; i < m->n_real; ++i) {
        double invA = 1. / m->area[i];
        for (int k = 0; k < V; ++k) { gx[V * i + k] *= invA; gy[V * i + k] *= invA; }
    }
    for (int64_t i = m->n_real; i < m->n_total; ++i)
        for (int k = 0; k < V; ++k) { gx[V * i + k] = 0.; gy[V * i + k] = 0.; }
}

/* Min/max + smooth-switch limiter, explicit.cpp:174-258 (K from ph->K; the
 * reference hard-codes K = 7.5 at explicit.cpp:27). */
void fvo_calc_limiters(const fvo_mesh* m, const fvo_physics* ph, const double* q, const double* gx,
                       const double* gy, double* lim) {
    const int V = ph->V;
    const size_t n = (size_t)V * m->n_total;
    double* qmin = malloc(n * 8);
    double* qmax = malloc(n * 8);
    for (size_t i = 0; i < n; ++i) { lim[i] = 1.; qmin[i] = q[i]; qmax[i] = q[i]; }
    for (int64_t e = 0; e < m->n_edges; ++e) {
        uint32_t i = m->edge_cells[2 * e], j = m->edge_cells[2 * e + 1];
        for (int k = 0; k < V; ++k) {
            qmin[V * i + k] = dmin(qmin[V * i + k], q[V * j + k]);
            qmin[V * j + k] = dmin(qmin[V * j + k], q[V * i + k]);
            qmax[V * i + k] = dmax(qmax[V * i + k], q[V * j + k]);
            qmax[V * j + k] = dmax(qmax[V * j + k], q[V * i + k]);
        }
    }
    const double tol = 1e-15;
    for (int64_t e = 0; e < m->n_edges; ++e) {
        uint32_t ids[2] = {m->edge_cells[2 * e], m->edge_cells[2 * e + 1]};
        for (int s = 0; s < 2; ++s) {
            uint32_t id = ids[s];
            if (id >= (uint64_t)m->n_real) continue;
            double dx = m->ecx[e] - m->ccx[id], dy = m->ecy[e] - m->ccy[id];
            double sqrt_area = sqrt(m->area[id]);
            for (int k = 0; k < V; ++k) {
                double dqg = gx[V * id + k] * dx + gy[V * id + k] * dy;
                double delta_max = qmax[V * id + k] - q[V * id + k];
                double delta_min = qmin[V * id + k] - q[V * id + k];
                const double Ka = ph->K * sqrt_area;
                const double K3a = Ka * Ka * Ka;
                const double d2 = (delta_max - delta_min) * (delta_max - delta_min);
                double sig;
                if (d2 <= K3a) sig = 1.;
                else if (d2 <= 2 * K3a) {
                    double y = (d2 / K3a - 1.0);
                    sig = 2.0 * y * y * y - 3.0 * y * y + 1.0;
                } else sig = 0.;
                double l = 1.0;
                if (sig < 1.0) {
                    if (dqg > tol) l = fvo_limiter_func(ph, delta_max / dqg);
                    else if (dqg < -tol) l = fvo_limiter_func(ph, delta_min / dqg);
                    else l = 1.0;
                }
                l = sig + (1.0 - sig) * l;
                lim[V * id + k] = dmin(lim[V * id + k], l);
            }
        }
    }
    free(qmin); free(qmax);
}

/* Optional positivity guard (an extension, not in the reference): a
 * reconstructed Euler face state with non-positive density or pressure is
 * replaced by the cell value. */
static void guard_face(const fvo_physics* ph, double* qf, const double* qc) {
    if (!ph->positivity_guard || ph->V != 4) return;
    const double p = (ph->gamma - 1) * (qf[3] - 0.5 / qf[0] * (qf[1] * qf[1] + qf[2] * qf[2]));
    if (!(qf[0] > 0.) || !(p > 0.))
        for (int k = 0; k < 4; ++k) qf[k] = qc[k];
}

/* Face gradient for the diffusive fluxes, explicit.cpp:70-109: the mean of
 * the two cell gradients with its component along the centroid line replaced
 * by the centroid difference quotient (cell states, not face states). */
static void face_gradient(int V, double* gxf, double* gyf, const double* gxi, const double* gyi,
                          const double* gxj, const double* gyj, const double* qi, const double* qj,
                          const double* ci, const double* cj) {
    double t0 = ci[0] - cj[0], t1 = ci[1] - cj[1];
    const double lij = sqrt(t0 * t0 + t1 * t1);
    t0 = t0 / lij;
    t1 = t1 / lij;
    for (int k = 0; k < V; ++k) {
        const double dir = (qi[k] - qj[k]) / lij;
        const double bx = (gxi[k] + gxj[k]) * 0.5, by = (gyi[k] + gyj[k]) * 0.5;
        const double dot = bx * t0 + by * t1;
        gxf[k] = bx - (dot - dir) * t0;
        gyf[k] = by - (dot - dir) * t1;
    }
}

/* Edge flux loop, explicit.cpp:261-364. */
void fvo_calc_time_derivatives(const fvo_mesh* m, const fvo_physics* ph, const double* q,
                               const double* gx, const double* gy, const double* lim, double* qt) {
    const int V = ph->V;
    memset(qt, 0, sizeof(double) * V * m->n_total);
    double qi[8], qj[8], f[8], n[2], gxf[8], gyf[8];
    for (int64_t e = 0; e < m->n_edges; ++e) {
        uint32_t i = m->edge_cells[2 * e], j = m->edge_cells[2 * e + 1];
        double le = m->elen[e];
        n[0] = m->enx[e]; n[1] = m->eny[e];
        double cx = m->ecx[e], cy = m->ecy[e];
        double di0 = cx - m->ccx[i], di1 = cy - m->ccy[i];
        double dj0 = cx - m->ccx[j], dj1 = cy - m->ccy[j];
        if (ph->order2) {
            for (int k = 0; k < V; ++k) {
                size_t ki = (size_t)V * i + k, kj = (size_t)V * j + k;
                qi[k] = q[ki] + (gx[ki] * di0 + gy[ki] * di1) * lim[ki];
                qj[k] = q[kj] + (gx[kj] * dj0 + gy[kj] * dj1) * lim[kj];
            }
            guard_face(ph, qi, q + (size_t)V * i);
            guard_face(ph, qj, q + (size_t)V * j);
        } else {
            for (int k = 0; k < V; ++k) { qi[k] = q[(size_t)V * i + k]; qj[k] = q[(size_t)V * j + k]; }
        }
        if (ph->diffusive) {
            const double ci[2] = {m->ccx[i], m->ccy[i]}, cj[2] = {m->ccx[j], m->ccy[j]};
            face_gradient(V, gxf, gyf, gx + (size_t)V * i, gy + (size_t)V * i, gx + (size_t)V * j,
                          gy + (size_t)V * j, q + (size_t)V * i, q + (size_t)V * j, ci, cj);
        }
        if (!ph->diffusive)  /* gxv = gyv = 0, explicit.cpp:332-337 */
            for (int k = 0; k < V; ++k) { gxf[k] = 0.; gyf[k] = 0.; }
        /* examples/heatTransfer/main.cpp:63-73, flatPlate/main.cpp:126-225 */
        fvo_flux_grad(ph, f, qi, qj, gxf, gyf, n);
        for (int k = 0; k < V; ++k) {
            qt[(size_t)V * i + k] -= f[k] * le / m->area[i];
            qt[(size_t)V * j + k] += f[k] * le / m->area[j];
        }
    }
    for (int64_t i = m->n_real; i < m->n_total; ++i)
        for (int k = 0; k < V; ++k) qt[(size_t)V * i + k] = 0.;
}

/* Ghost fill, explicit.cpp:380-417. */
void fvo_update_bounds(const fvo_mesh* m, const fvo_physics* ph, double* q, const double* gx,
                       const double* gy, const double* lim) {
    const int V = ph->V;
    double qint[8], n[2];
    for (int64_t b = 0; b < m->n_bound; ++b) {
        uint32_t e = m->bound_edges[b];
        n[0] = m->enx[e]; n[1] = m->eny[e];
        uint32_t ii = m->edge_cells[2 * e], ib = m->edge_cells[2 * e + 1];
        if (ph->order2) {
            double d0 = m->ecx[e] - m->ccx[ii], d1 = m->ecy[e] - m->ccy[ii];
            for (int k = 0; k < V; ++k) {
                size_t kk = (size_t)V * ii + k;
                qint[k] = q[kk] + (gx[kk] * d0 + gy[kk] * d1) * lim[kk];
            }
            guard_face(ph, qint, q + (size_t)V * ii);
        } else {
            for (int k = 0; k < V; ++k) qint[k] = q[(size_t)V * ii + k];
        }
        bc_state(ph, m->bound_group[b], ph->ghost_bv ? ph->ghost_bv + 4 * (size_t)b : ph->group_bv + 4 * m->bound_group[b],
                 q + (size_t)V * ib, qint, n);
    }
}

/* Implicit residual smoothing, explicit.cpp:32-66: two Jacobi sweeps of
 * (1 + ne eps) r_i - eps sum_j r_j = qt_i (eps = 0.6, ne = 3 or 4 faces), the
 * neighbour sums accumulated in edge order; ghosts keep qt = 0. */
void fvo_smooth_residuals(const fvo_mesh* m, const fvo_physics* ph, double* qt) {
    const int V = ph->V;
    const double epsilon = 0.6;
    const size_t n = (size_t)V * m->n_total;
    double* qt0 = malloc(n * 8);
    double* s = malloc(n * 8);
    int* ne = calloc((size_t)m->n_total, sizeof(int));
    for (int64_t e = 0; e < m->n_edges; ++e) { ne[m->edge_cells[2 * e]]++; ne[m->edge_cells[2 * e + 1]]++; }
    memcpy(qt0, qt, n * 8);
    for (int it = 0; it < 2; ++it) {
        for (size_t i = 0; i < n; ++i) s[i] = 0.;
        for (int64_t e = 0; e < m->n_edges; ++e) {
            uint32_t i = m->edge_cells[2 * e], j = m->edge_cells[2 * e + 1];
            for (int k = 0; k < V; ++k) {
                s[(size_t)V * i + k] -= qt[(size_t)V * j + k] * epsilon;
                s[(size_t)V * j + k] -= qt[(size_t)V * i + k] * epsilon;
            }
        }
        for (int64_t i = 0; i < m->n_real; ++i) {
            const double nf = ne[i] == 3 ? 3 : 4;  /* cellsIsTriangle ? 3 : 4 */
            for (int k = 0; k < V; ++k)
                qt[(size_t)V * i + k] = (qt0[(size_t)V * i + k] - s[(size_t)V * i + k]) / (1. + nf * epsilon);
        }
    }
    free(qt0); free(s); free(ne);
}

/* Residual norms, explicit.cpp:481-496 (single rank). */
void fvo_calc_residuals(const fvo_mesh* m, const fvo_physics* ph, const double* qt, double* R) {
    const int V = ph->V;
    for (int k = 0; k < V; ++k) R[k] = 0.;
    for (int64_t i = 0; i < m->n_real; ++i)
        for (int k = 0; k < V; ++k) R[k] += qt[(size_t)V * i + k] * qt[(size_t)V * i + k] * m->area[i];
    for (int k = 0; k < V; ++k) R[k] = sqrt(R[k]);
}

/* Body of run(), explicit.cpp:665-801, with the RK coefficients as input
 * (the reference hard-codes the 5-stage set at explicit.cpp:681-687). */
int fvo_run_loop(const fvo_mesh* m, const fvo_physics* ph, double* q, const double* alpha,
                 int n_alpha, uint64_t max_step, double max_time, double tolerance,
                 uint64_t print_interval, uint64_t* out_step, double* out_time, double* out_R,
                 double* out_qt) {
    const int V = ph->V;
    const size_t n = (size_t)V * m->n_total;
    double* qk = calloc(n, 8); double* qt = calloc(n, 8); double* gx = calloc(n, 8);
    double* gy = calloc(n, 8); double* lim = calloc(n, 8); double* dt = calloc(m->n_total, 8);
    double R0[8], R[8];
    for (int k = 0; k < V; ++k) R[k] = 1.0;
    uint64_t step = 0;
    double time = 0;
    fvo_update_bounds(m, ph, q, gx, gy, lim);
    for (;;) {
        double Rmax = 0.0;
        if (step > 0) { for (int k = 0; k < V; ++k) Rmax = dmax(R[k], Rmax); }
        else Rmax = 1.0;
        if ((step >= max_step) | (time >= max_time) | (Rmax < tolerance)) break;
        fvo_calc_dt(m, ph, q, dt);
        if (ph->global_dt) fvo_min_dt(m, dt);
        memcpy(qk, q, n * 8);
        for (int s = 0; s < n_alpha; ++s) {
            if (ph->order2 || ph->diffusive) fvo_calc_gradients(m, ph, qk, gx, gy);
            if (ph->order2) fvo_calc_limiters(m, ph, qk, gx, gy, lim);
            fvo_calc_time_derivatives(m, ph, qk, gx, gy, lim, qt);
            if (ph->smooth) fvo_smooth_residuals(m, ph, qt);  /* explicit.cpp:743 */
            for (int64_t i = 0; i < m->n_total; ++i) /* update_cells, explicit.cpp:368-378 */
                for (int k = 0; k < V; ++k) {
                    size_t kk = (size_t)V * i + k;
                    qk[kk] = q[kk] + qt[kk] * dt[i] * alpha[s];
                }
            fvo_update_bounds(m, ph, qk, gx, gy, lim);
        }
        memcpy(q, qk, n * 8);
        if (step == 0) {
            fvo_calc_residuals(m, ph, qt, R0);
            for (int k = 0; k < V; ++k) R[k] = R0[k];
        } else if ((step % print_interval == 0) | (tolerance > 1.01e-16)) {
            fvo_calc_residuals(m, ph, qt, R);
            for (int k = 0; k < V; ++k) R[k] = R[k] / R0[k];
        }
        step += 1;
        time += dt[0];
    }
    if (out_step) *out_step = step;
    if (out_time) *out_time = time;
    if (out_R) memcpy(out_R, R, V * 8);
    if (out_qt) memcpy(out_qt, qt, n * 8);
    free(qk); free(qt); free(gx); free(gy); free(lim); free(dt);
    return 0;
}

void fvo_boundary_force(const fvo_mesh* m, const fvo_physics* ph, const double* q, int group,
                        double* fx, double* fy) {
    const int V = ph->V;
    const double gm1 = ph->gamma - 1;
    double sx = 0., sy = 0.;
    for (int64_t b = 0; b < m->n_bound; ++b) {
        if (m->bound_group[b] != group) continue;
        uint32_t e = m->bound_edges[b];
        uint32_t ii = m->edge_cells[2 * e];
        double p = pres(gm1, q + (size_t)V * ii);
        sx += p * m->enx[e] * m->elen[e];
        sy += p * m->eny[e] * m->elen[e];
    }
    *fx = sx; *fy = sy;
}
