/*
 * qsv_oracle.c — TEST INFRASTRUCTURE ONLY (the parity checker; never linked into the
 * product library).  A scalar CPU restatement of the reference statevector path:
 *
 *   or_apply             <- QarpSimulator::apply_command   qarp_simulator.cpp:356-596
 *                           (csim per-gate kernels, third_party/csim/update_ops_*.cpp;
 *                            apply_dense_k, src/simulator/dense_kernel.cpp:23-81)
 *   or_transition        <- explicit_transition oracle, src/qarpx/tests/test_expectation_kernel.cpp:22-49
 *                           (same value pauli_transition, pauli_expectation.cpp:159-167, computes)
 *   or_apply_observable  <- apply_observable                qarp_simulator.cpp:1459-1479
 *   or_uniforms/or_sample<- sample_terminal                 qarp_simulator.cpp:751-783 with the
 *                           toolchain's std::mt19937 / std::generate_canonical<double,53> /
 *                           std::discrete_distribution (libstdc++ bits/random.tcc)
 *   or_adjoint(_phi)     <- run_gradient_core               qarp_simulator.cpp:1519-1605,
 *                           apply_generator :1352-1418, Command::dagger src/core/command.cpp:19-59
 *
 * Plain C99, one thread, no fusion: every command is one pass, as the reference's
 * unfused apply loop.  The packed command format is include/qsv.h's.
 */
#include "qsv_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define OR_PI 3.14159265358979323846

typedef double complex cplx;

static _Thread_local char g_err[512];
const char* or_last_error(void) { return g_err; }

static int fail(int code, const char* msg) {
    snprintf(g_err, sizeof g_err, "%s", msg);
    return code;
}

/* gate codes: qarpx::GateType enumerator order (src/qarpx/include/qarpx/core/gates.h:8-58) */
enum {
    G_X = 0, G_Y, G_Z, G_H, G_S, G_SDG, G_T, G_TDG, G_SX, G_SXDG, G_ID,
    G_RX, G_RY, G_RZ, G_P, G_U,
    G_CX, G_CY, G_CZ, G_SWAP, G_ECR, G_ISWAP, G_ISWAPDG,
    G_CH, G_CS, G_CSDG, G_CSX, G_CSXDG,
    G_CRX, G_CRY, G_CRZ, G_CP, G_RZZ, G_RXX, G_RYY,
    G_CU, G_CCX, G_CSWAP, G_MCZ, G_GPHASE,
    G_BARRIER, G_MEASURE, G_RESET, G_BBEGIN, G_BELSE, G_BEND, G_CUSTOM,
    /* structured-program records of include/qsv.h */
    G_PERMUTATION = 200, G_CTRL_UNITARY = 201
};

/* ---------------------------------------------------------------- command decoding */

typedef struct {
    int gate, nq, np, ncb, flags;
    const uint32_t* q;
    const double* p;
    const double* m;   /* Custom / controlled-unitary matrix (interleaved) or NULL */
    const uint64_t* t; /* permutation table or NULL */
    size_t size;       /* bytes of the record */
} rec_t;

static int decode(const uint8_t* buf, size_t nbytes, size_t off, rec_t* r) {
    if (off + 8 > nbytes) return fail(1, "command buffer truncated (header)");
    uint16_t gate; memcpy(&gate, buf + off, 2);
    r->gate = gate;
    r->nq = buf[off + 2]; r->np = buf[off + 3]; r->ncb = buf[off + 4]; r->flags = buf[off + 5];
    const int ncond = buf[off + 6];   /* condition entries: bits then values, after the cbits */
    size_t o = off + 8;
    r->q = (const uint32_t*)(buf + o);
    o += 4u * (size_t)(r->nq + r->ncb + 2 * ncond);
    if (ncond) r->flags |= 1;
    o = (o + 7u) & ~(size_t)7u;
    r->p = (const double*)(buf + o);
    o += 8u * (size_t)r->np;
    r->m = NULL;
    r->t = NULL;
    if (r->gate == G_CUSTOM) {
        if (r->nq < 1 || r->nq > 8) return fail(2, "Custom gate must carry 1..8 qubit targets");
        r->m = (const double*)(buf + o);
        o += 16u * ((size_t)1 << (2 * r->nq));
    } else if (r->gate == G_PERMUTATION) {
        if (r->nq < 1 || r->nq > 26) return fail(1, "permutation must act on 1..26 qubits");
        r->t = (const uint64_t*)(buf + o);
        o += 8u * ((size_t)1 << r->nq);
    } else if (r->gate == G_CTRL_UNITARY) {
        if (r->nq < 2 || r->nq > 13) return fail(1, "controlled unitary must act on 1..12 targets + 1 control");
        r->m = (const double*)(buf + o);
        o += 16u * ((size_t)1 << (2 * (r->nq - 1)));
    }
    if (o > nbytes) return fail(1, "command buffer truncated (payload)");
    r->size = o - off;
    return 0;
}

/* ---------------------------------------------------------------- primitive kernels */

/* 2x2 matrix (row-major) on target t: pairs (i0, i0 | 2^t) */
static void k_single(cplx* s, int n, uint32_t t, const cplx m[4]) {
    const uint64_t dim = 1ull << n, bit = 1ull << t;
    for (uint64_t i = 0; i < dim; ++i) {
        if (i & bit) continue;
        cplx a0 = s[i], a1 = s[i | bit];
        s[i] = m[0] * a0 + m[1] * a1;
        s[i | bit] = m[2] * a0 + m[3] * a1;
    }
}

/* 2x2 matrix on target t where every control bit is 1 */
static void k_controlled(cplx* s, int n, uint64_t cmask, uint32_t t, const cplx m[4]) {
    const uint64_t dim = 1ull << n, bit = 1ull << t;
    for (uint64_t i = 0; i < dim; ++i) {
        if ((i & bit) || (i & cmask) != cmask) continue;
        cplx a0 = s[i], a1 = s[i | bit];
        s[i] = m[0] * a0 + m[1] * a1;
        s[i | bit] = m[2] * a0 + m[3] * a1;
    }
}

static void k_swap(cplx* s, int n, uint32_t a, uint32_t b) {
    const uint64_t dim = 1ull << n, ba = 1ull << a, bb = 1ull << b;
    for (uint64_t i = 0; i < dim; ++i)
        if ((i & ba) && !(i & bb)) {
            uint64_t j = (i & ~ba) | bb;
            cplx tmp = s[i]; s[i] = s[j]; s[j] = tmp;
        }
}

/* P|i> = i^{nY} (-1)^{popcount(i & z)} |i ^ x> */
static cplx pauli_phase(uint64_t i, uint64_t x, uint64_t z) {
    static const cplx ipow[4] = {1.0, I, -1.0, -I};
    int ny = __builtin_popcountll(x & z);
    cplx ph = ipow[ny & 3];
    return (__builtin_popcountll(i & z) & 1) ? -ph : ph;
}

/* exp(-i theta/2 P) */
static void k_pauli_rot(cplx* s, int n, uint64_t x, uint64_t z, double theta) {
    const uint64_t dim = 1ull << n;
    const double c = cos(theta / 2.0), sn = sin(theta / 2.0);
    if (x == 0) {
        for (uint64_t i = 0; i < dim; ++i) {
            double sign = (__builtin_popcountll(i & z) & 1) ? -1.0 : 1.0;
            s[i] *= (c - I * (sign * sn));
        }
        return;
    }
    const uint64_t pivot = x & (~x + 1);  /* lowest flipped bit */
    for (uint64_t i = 0; i < dim; ++i) {
        if (i & pivot) continue;
        uint64_t j = i ^ x;
        cplx ai = s[i], aj = s[j];
        /* (P psi)[i] = phase(j) psi[j];  (P psi)[j] = phase(i) psi[i] */
        s[i] = c * ai - I * sn * pauli_phase(j, x, z) * aj;
        s[j] = c * aj - I * sn * pauli_phase(i, x, z) * ai;
    }
}

static void k_dense(cplx* s, int n, int k, const uint32_t* qubits, const double* mat) {
    const int D = 1 << k;
    uint32_t sorted[8];
    for (int b = 0; b < k; ++b) sorted[b] = qubits[b];
    for (int a = 0; a < k; ++a)
        for (int b = a + 1; b < k; ++b)
            if (sorted[b] < sorted[a]) { uint32_t t = sorted[a]; sorted[a] = sorted[b]; sorted[b] = t; }
    uint64_t masks[256];
    for (int l = 0; l < D; ++l) {
        uint64_t mk = 0;
        for (int b = 0; b < k; ++b) if ((l >> b) & 1) mk |= 1ull << qubits[b];
        masks[l] = mk;
    }
    cplx in[256];
    const uint64_t outer = (1ull << n) >> k;
    for (uint64_t o = 0; o < outer; ++o) {
        uint64_t base = o;
        for (int b = 0; b < k; ++b) {
            uint64_t p = sorted[b];
            uint64_t low = base & ((1ull << p) - 1);
            base = ((base >> p) << (p + 1)) | low;
        }
        for (int l = 0; l < D; ++l) in[l] = s[base | masks[l]];
        for (int y = 0; y < D; ++y) {
            cplx acc = 0.0;
            for (int x = 0; x < D; ++x) {
                const double* e = mat + 2 * (y * D + x);
                acc += (e[0] + I * e[1]) * in[x];
            }
            s[base | masks[y]] = acc;
        }
    }
}

/* |x> -> |table[x]> on qubits[0..k), out of place then copied back
 * (apply_permutation, src/qarpx/src/simulator/program.cpp:610-643) */
static int k_permutation(cplx* s, int n, int k, const uint32_t* qubits, const uint64_t* table) {
    const uint64_t dim = 1ull << n;
    uint64_t keep = ~0ull;
    for (int b = 0; b < k; ++b) keep &= ~(1ull << qubits[b]);
    cplx* out = (cplx*)malloc(dim * sizeof(cplx));
    if (!out) return fail(2, "out of memory");
    for (uint64_t i = 0; i < dim; ++i) {
        uint64_t x = 0, j = i & keep;
        for (int b = 0; b < k; ++b) x |= ((i >> qubits[b]) & 1ull) << b;
        const uint64_t y = table[x];
        for (int b = 0; b < k; ++b) j |= ((y >> b) & 1ull) << qubits[b];
        out[j] = s[i];
    }
    memcpy(s, out, dim * sizeof(cplx));
    free(out);
    return 0;
}

/* one (control, power) step of apply_controlled_powers (program.cpp:680-708): the m-target
 * matrix on every group whose control bit is set */
static int k_controlled_dense(cplx* s, int n, int m, const uint32_t* targets, uint32_t control,
                              const double* mat) {
    const uint64_t d = 1ull << m, cbit = 1ull << control;
    uint32_t sorted[16];
    for (int b = 0; b < m; ++b) sorted[b] = targets[b];
    for (int a = 0; a < m; ++a)
        for (int b = a + 1; b < m; ++b)
            if (sorted[b] < sorted[a]) { uint32_t t = sorted[a]; sorted[a] = sorted[b]; sorted[b] = t; }
    uint64_t* off = (uint64_t*)malloc(d * sizeof(uint64_t));
    cplx* col = (cplx*)malloc(d * sizeof(cplx));
    if (!off || !col) { free(off); free(col); return fail(2, "out of memory"); }
    for (uint64_t l = 0; l < d; ++l) {
        uint64_t o = 0;
        for (int b = 0; b < m; ++b) if ((l >> b) & 1) o |= 1ull << targets[b];
        off[l] = o;
    }
    const uint64_t outer = (1ull << n) >> m;
    for (uint64_t o = 0; o < outer; ++o) {
        uint64_t base = o;
        for (int b = 0; b < m; ++b) {
            const uint64_t p = sorted[b];
            base = ((base >> p) << (p + 1)) | (base & ((1ull << p) - 1));
        }
        if (!(base & cbit)) continue;
        for (uint64_t l = 0; l < d; ++l) col[l] = s[base | off[l]];
        for (uint64_t y = 0; y < d; ++y) {
            cplx acc = 0.0;
            for (uint64_t x = 0; x < d; ++x) {
                const double* e = mat + 2 * (y * d + x);
                acc += (e[0] + I * e[1]) * col[x];
            }
            s[base | off[y]] = acc;
        }
    }
    free(off);
    free(col);
    return 0;
}

/* ---------------------------------------------------------------- gate matrices */

static void mat_rx(double th, cplx m[4]) {  /* exp(-i th/2 X) */
    double c = cos(th / 2.0), sn = sin(th / 2.0);
    m[0] = c; m[1] = -I * sn; m[2] = -I * sn; m[3] = c;
}
static void mat_ry(double th, cplx m[4]) {
    double c = cos(th / 2.0), sn = sin(th / 2.0);
    m[0] = c; m[1] = -sn; m[2] = sn; m[3] = c;
}
static void mat_rz(double th, cplx m[4]) {
    double c = cos(th / 2.0), sn = sin(th / 2.0);
    m[0] = c - I * sn; m[1] = 0; m[2] = 0; m[3] = c + I * sn;
}
static void mat_p(double th, cplx m[4]) {
    m[0] = 1; m[1] = 0; m[2] = 0; m[3] = cos(th) + I * sin(th);
}
/* OpenQASM 3 U(theta, phi, lambda) (qarp_simulator.cpp:524-537) */
static void mat_u(double th, double ph, double la, cplx m[4]) {
    double c = cos(th / 2.0), sn = sin(th / 2.0);
    m[0] = c;
    m[1] = -(cos(la) + I * sin(la)) * sn;
    m[2] = (cos(ph) + I * sin(ph)) * sn;
    m[3] = (cos(ph + la) + I * sin(ph + la)) * c;
}

static void fixed_matrix(int gate, cplx m[4]) {
    const double r = 1.0 / sqrt(2.0);
    memset(m, 0, 4 * sizeof(cplx));
    switch (gate) {
        case G_X: m[1] = 1; m[2] = 1; break;
        case G_Y: m[1] = -I; m[2] = I; break;
        case G_Z: m[0] = 1; m[3] = -1; break;
        case G_H: m[0] = r; m[1] = r; m[2] = r; m[3] = -r; break;
        case G_S: m[0] = 1; m[3] = I; break;
        case G_SDG: m[0] = 1; m[3] = -I; break;
        case G_T: m[0] = 1; m[3] = cos(OR_PI / 4) + I * sin(OR_PI / 4); break;
        case G_TDG: m[0] = 1; m[3] = cos(-OR_PI / 4) + I * sin(-OR_PI / 4); break;
        case G_SX: m[0] = 0.5 + 0.5 * I; m[1] = 0.5 - 0.5 * I; m[2] = 0.5 - 0.5 * I; m[3] = 0.5 + 0.5 * I; break;
        case G_SXDG: m[0] = 0.5 - 0.5 * I; m[1] = 0.5 + 0.5 * I; m[2] = 0.5 + 0.5 * I; m[3] = 0.5 - 0.5 * I; break;
        default: m[0] = 1; m[3] = 1; break;
    }
}

/* ---------------------------------------------------------------- apply_command */

static int apply_rec(cplx* s, int n, const rec_t* r);

static int apply_simple(cplx* s, int n, int gate, const uint32_t* q, const double* p) {
    rec_t r; memset(&r, 0, sizeof r);
    r.gate = gate; r.q = q; r.p = p;
    r.nq = (gate >= G_CX && gate <= G_RYY) ? 2 : 1;
    r.np = (gate == G_RZ) ? 1 : 0;
    return apply_rec(s, n, &r);
}

static int need_params(const rec_t* r, int k) {
    if (r->np < k) return fail(2, "gate is missing a parameter");
    return 0;
}

static int apply_rec(cplx* s, int n, const rec_t* r) {
    const uint64_t dim = 1ull << n;
    const int g = r->gate;
    for (int b = 0; b < r->nq; ++b)
        if ((int)r->q[b] >= n) return fail(1, "command acts on a qubit outside the register");
    cplx m[4];
    switch (g) {
        case G_X: case G_Y: case G_Z: case G_H: case G_S: case G_SDG: case G_T: case G_TDG:
        case G_SX: case G_SXDG:
            fixed_matrix(g, m); k_single(s, n, r->q[0], m); return 0;
        case G_ID: case G_BARRIER: case G_MEASURE: case G_RESET: return 0;
        case G_RX: if (need_params(r, 1)) return 2; mat_rx(r->p[0], m); k_single(s, n, r->q[0], m); return 0;
        case G_RY: if (need_params(r, 1)) return 2; mat_ry(r->p[0], m); k_single(s, n, r->q[0], m); return 0;
        case G_RZ: if (need_params(r, 1)) return 2; mat_rz(r->p[0], m); k_single(s, n, r->q[0], m); return 0;
        case G_P:  if (need_params(r, 1)) return 2; mat_p(r->p[0], m); k_single(s, n, r->q[0], m); return 0;
        case G_U:  if (need_params(r, 3)) return 2; mat_u(r->p[0], r->p[1], r->p[2], m); k_single(s, n, r->q[0], m); return 0;
        case G_CX: case G_CY: case G_CZ: case G_CH: case G_CS: case G_CSDG: case G_CSX: case G_CSXDG: {
            static const int tgt[] = {G_X, G_Y, G_Z};
            int base = g == G_CX ? G_X : g == G_CY ? G_Y : g == G_CZ ? G_Z : g == G_CH ? G_H
                     : g == G_CS ? G_S : g == G_CSDG ? G_SDG : g == G_CSX ? G_SX : G_SXDG;
            (void)tgt;
            fixed_matrix(base, m);
            k_controlled(s, n, 1ull << r->q[0], r->q[1], m);
            return 0;
        }
        case G_SWAP: k_swap(s, n, r->q[0], r->q[1]); return 0;
        case G_ECR: {  /* decompose_ecr, src/transpiler/decompositions.cpp:391-404 */
            const uint32_t q0 = r->q[0], q1 = r->q[1];
            const uint32_t c01[2] = {q0, q1};
            const double pp = OR_PI / 4, pm = -OR_PI / 4;
            apply_simple(s, n, G_H, &q1, NULL);
            apply_simple(s, n, G_CX, c01, NULL);
            apply_simple(s, n, G_RZ, &q1, &pp);
            apply_simple(s, n, G_CX, c01, NULL);
            apply_simple(s, n, G_X, &q0, NULL);
            apply_simple(s, n, G_CX, c01, NULL);
            apply_simple(s, n, G_RZ, &q1, &pm);
            apply_simple(s, n, G_CX, c01, NULL);
            apply_simple(s, n, G_H, &q1, NULL);
            return 0;
        }
        case G_ISWAP: {  /* decompose_iswap, decompositions.cpp:407-417 */
            const uint32_t q0 = r->q[0], q1 = r->q[1];
            const uint32_t c01[2] = {q0, q1}, c10[2] = {q1, q0};
            apply_simple(s, n, G_S, &q0, NULL);
            apply_simple(s, n, G_S, &q1, NULL);
            apply_simple(s, n, G_H, &q0, NULL);
            apply_simple(s, n, G_CX, c01, NULL);
            apply_simple(s, n, G_CX, c10, NULL);
            apply_simple(s, n, G_H, &q1, NULL);
            return 0;
        }
        case G_ISWAPDG: {  /* decompose_iswapdg, decompositions.cpp:421-431 */
            const uint32_t q0 = r->q[0], q1 = r->q[1];
            const uint32_t c01[2] = {q0, q1}, c10[2] = {q1, q0};
            apply_simple(s, n, G_H, &q1, NULL);
            apply_simple(s, n, G_CX, c10, NULL);
            apply_simple(s, n, G_CX, c01, NULL);
            apply_simple(s, n, G_H, &q0, NULL);
            apply_simple(s, n, G_SDG, &q1, NULL);
            apply_simple(s, n, G_SDG, &q0, NULL);
            return 0;
        }
        case G_CRX: case G_CRY: case G_CRZ: case G_CP:
            if (need_params(r, 1)) return 2;
            if (g == G_CRX) mat_rx(r->p[0], m);
            else if (g == G_CRY) mat_ry(r->p[0], m);
            else if (g == G_CRZ) mat_rz(r->p[0], m);
            else mat_p(r->p[0], m);
            k_controlled(s, n, 1ull << r->q[0], r->q[1], m);
            return 0;
        case G_RZZ: case G_RXX: case G_RYY: {
            if (need_params(r, 1)) return 2;
            uint64_t b = (1ull << r->q[0]) | (1ull << r->q[1]);
            uint64_t x = (g == G_RZZ) ? 0 : b;
            uint64_t z = (g == G_RXX) ? 0 : b;
            k_pauli_rot(s, n, x, z, r->p[0]);
            return 0;
        }
        case G_CU: {
            if (need_params(r, 4)) return 2;
            mat_u(r->p[0], r->p[1], r->p[2], m);
            cplx ph = cos(r->p[3]) + I * sin(r->p[3]);
            for (int e = 0; e < 4; ++e) m[e] *= ph;
            k_controlled(s, n, 1ull << r->q[0], r->q[1], m);
            return 0;
        }
        case G_CCX:
            if (r->nq < 3) return fail(2, "CCX requires 3 qubits");
            fixed_matrix(G_X, m);
            k_controlled(s, n, (1ull << r->q[0]) | (1ull << r->q[1]), r->q[2], m);
            return 0;
        case G_CSWAP: {  /* CX(t1,t0) CCX(c,t0,t1) CX(t1,t0), qarp_simulator.cpp:487-503 */
            if (r->nq < 3) return fail(2, "CSWAP requires 3 qubits");
            const uint32_t c = r->q[0], t0 = r->q[1], t1 = r->q[2];
            fixed_matrix(G_X, m);
            k_controlled(s, n, 1ull << t1, t0, m);
            k_controlled(s, n, (1ull << c) | (1ull << t0), t1, m);
            k_controlled(s, n, 1ull << t1, t0, m);
            return 0;
        }
        case G_MCZ: {
            if (r->nq < 2) return fail(2, "MCZ requires >=2 qubits");
            uint64_t cm = 0;
            for (int b = 0; b < r->nq - 1; ++b) cm |= 1ull << r->q[b];
            fixed_matrix(G_Z, m);
            k_controlled(s, n, cm, r->q[r->nq - 1], m);
            return 0;
        }
        case G_GPHASE: {
            if (need_params(r, 1)) return 2;
            cplx ph = cos(r->p[0]) + I * sin(r->p[0]);
            for (uint64_t i = 0; i < dim; ++i) s[i] *= ph;
            return 0;
        }
        case G_CUSTOM:
            if (r->nq == 1) {
                for (int e = 0; e < 4; ++e) m[e] = r->m[2 * e] + I * r->m[2 * e + 1];
                k_single(s, n, r->q[0], m);
            } else {
                k_dense(s, n, r->nq, r->q, r->m);
            }
            return 0;
        case G_PERMUTATION:
            return k_permutation(s, n, r->nq, r->q, r->t);
        case G_CTRL_UNITARY:
            return k_controlled_dense(s, n, r->nq - 1, r->q, r->q[r->nq - 1], r->m);
        default:
            return fail(2, "unsupported gate");
    }
}

int or_apply(double* state, int n, const uint8_t* cmds, size_t nbytes) {
    size_t off = 0;
    while (off < nbytes) {
        rec_t r;
        int rc = decode(cmds, nbytes, off, &r);
        if (rc) return rc;
        rc = apply_rec((cplx*)state, n, &r);
        if (rc) return rc;
        off += r.size;
    }
    return 0;
}

/* ---------------------------------------------------------------- dagger / generator */

/* Command::dagger (src/core/command.cpp:19-59) applied in place to a copy of the record */
static int apply_dagger(cplx* s, int n, const rec_t* r) {
    rec_t d = *r;
    double p[4];
    static double mbuf[2 * 65536];
    switch (r->gate) {
        case G_S: d.gate = G_SDG; break;
        case G_SDG: d.gate = G_S; break;
        case G_T: d.gate = G_TDG; break;
        case G_TDG: d.gate = G_T; break;
        case G_SX: d.gate = G_SXDG; break;
        case G_SXDG: d.gate = G_SX; break;
        case G_ISWAP: d.gate = G_ISWAPDG; break;
        case G_ISWAPDG: d.gate = G_ISWAP; break;
        case G_CS: d.gate = G_CSDG; break;
        case G_CSDG: d.gate = G_CS; break;
        case G_CSX: d.gate = G_CSXDG; break;
        case G_CSXDG: d.gate = G_CSX; break;
        case G_U:
            p[0] = -r->p[0]; p[1] = -r->p[2]; p[2] = -r->p[1];
            d.p = p; break;
        case G_CU:
            p[0] = -r->p[0]; p[1] = -r->p[2]; p[2] = -r->p[1]; p[3] = -r->p[3];
            d.p = p; break;
        case G_CUSTOM: {
            const int D = 1 << r->nq;
            for (int y = 0; y < D; ++y)
                for (int x = 0; x < D; ++x) {
                    mbuf[2 * (y * D + x)] = r->m[2 * (x * D + y)];
                    mbuf[2 * (y * D + x) + 1] = -r->m[2 * (x * D + y) + 1];
                }
            d.m = mbuf;
            break;
        }
        default:
            for (int i = 0; i < r->np && i < 4; ++i) p[i] = -r->p[i];
            d.p = p;
            break;
    }
    return apply_rec(s, n, &d);
}

/* apply_generator (qarp_simulator.cpp:1352-1418): state <- G state; returns prefactor */
static int apply_generator(cplx* s, int n, const rec_t* r, cplx* pref) {
    const uint64_t dim = 1ull << n;
    cplx m[4];
    const uint32_t q0 = r->nq > 0 ? r->q[0] : 0, q1 = r->nq > 1 ? r->q[1] : 0;
    switch (r->gate) {
        case G_RX: fixed_matrix(G_X, m); k_single(s, n, q0, m); *pref = -0.5 * I; return 1;
        case G_RY: fixed_matrix(G_Y, m); k_single(s, n, q0, m); *pref = -0.5 * I; return 1;
        case G_RZ: fixed_matrix(G_Z, m); k_single(s, n, q0, m); *pref = -0.5 * I; return 1;
        case G_P:
            for (uint64_t i = 0; i < dim; ++i) if (!(i & (1ull << q0))) s[i] = 0;
            *pref = I; return 1;
        case G_GPHASE: *pref = I; return 1;
        case G_CRX: case G_CRY: case G_CRZ:
            for (uint64_t i = 0; i < dim; ++i) if (!(i & (1ull << q0))) s[i] = 0;
            fixed_matrix(r->gate == G_CRX ? G_X : r->gate == G_CRY ? G_Y : G_Z, m);
            k_single(s, n, q1, m);
            *pref = -0.5 * I; return 1;
        case G_CP: {
            uint64_t both = (1ull << q0) | (1ull << q1);
            for (uint64_t i = 0; i < dim; ++i) if ((i & both) != both) s[i] = 0;
            *pref = I; return 1;
        }
        case G_RXX: case G_RYY: case G_RZZ: {
            int pg = r->gate == G_RXX ? G_X : r->gate == G_RYY ? G_Y : G_Z;
            fixed_matrix(pg, m);
            k_single(s, n, q0, m);
            k_single(s, n, q1, m);
            *pref = -0.5 * I; return 1;
        }
        default: return 0;
    }
}

/* ---------------------------------------------------------------- observables */

static int check_terms(int n, const uint64_t* xm, const uint64_t* zm, size_t nt) {
    const uint64_t lim = (n >= 64) ? ~0ull : ((1ull << n) - 1);
    for (size_t t = 0; t < nt; ++t)
        if (((xm[t] | zm[t]) & ~lim) != 0) return fail(1, "observable qubit out of range");
    return 0;
}

int or_transition(const double* bra, const double* ket, int n,
                  const uint64_t* xm, const uint64_t* zm, const double* coeff,
                  size_t nt, double out[2]) {
    if (n < 0 || n > 62) return fail(1, "n_qubits must be in [0, 62]");
    if (check_terms(n, xm, zm, nt)) return 1;
    const cplx* b = (const cplx*)bra;
    const cplx* k = (const cplx*)ket;
    const uint64_t dim = 1ull << n;
    cplx total = 0;
    for (size_t t = 0; t < nt; ++t) {
        cplx c = coeff[2 * t] + I * coeff[2 * t + 1];
        cplx acc = 0;
        for (uint64_t i = 0; i < dim; ++i)
            acc += conj(b[i ^ xm[t]]) * pauli_phase(i, xm[t], zm[t]) * k[i];
        total += c * acc;
    }
    out[0] = creal(total); out[1] = cimag(total);
    return 0;
}

int or_apply_observable(const double* psi, double* out, int n,
                        const uint64_t* xm, const uint64_t* zm, const double* coeff,
                        size_t nt) {
    if (check_terms(n, xm, zm, nt)) return 1;
    const uint64_t dim = 1ull << n;
    const cplx* p = (const cplx*)psi;
    cplx* o = (cplx*)out;
    for (uint64_t i = 0; i < dim; ++i) o[i] = 0;
    for (size_t t = 0; t < nt; ++t) {
        cplx c = coeff[2 * t] + I * coeff[2 * t + 1];
        for (uint64_t i = 0; i < dim; ++i)
            o[i ^ xm[t]] += c * pauli_phase(i, xm[t], zm[t]) * p[i];
    }
    return 0;
}

/* ---------------------------------------------------------------- sampling */

/* MT19937 (Matsumoto & Nishimura 1998), the std::mt19937 parameter set */
typedef struct { uint32_t mt[624]; int idx; } mt_t;

static void mt_seed(mt_t* g, uint32_t seed) {
    g->mt[0] = seed;
    for (int i = 1; i < 624; ++i)
        g->mt[i] = 1812433253u * (g->mt[i - 1] ^ (g->mt[i - 1] >> 30)) + (uint32_t)i;
    g->idx = 624;
}

static uint32_t mt_next(mt_t* g) {
    if (g->idx >= 624) {
        for (int i = 0; i < 624; ++i) {
            uint32_t y = (g->mt[i] & 0x80000000u) | (g->mt[(i + 1) % 624] & 0x7fffffffu);
            uint32_t v = g->mt[(i + 397) % 624] ^ (y >> 1);
            if (y & 1u) v ^= 0x9908b0dfu;
            g->mt[i] = v;
        }
        g->idx = 0;
    }
    uint32_t y = g->mt[g->idx++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

void or_uniforms(uint32_t seed, size_t n_shots, double* u) {
    mt_t g;
    mt_seed(&g, seed);
    for (size_t s = 0; s < n_shots; ++s) {
        /* generate_canonical<double, 53> with a 32-bit engine: two draws, sum in double */
        double sum = 0.0, tmp = 1.0;
        for (int k = 0; k < 2; ++k) {
            sum += (double)mt_next(&g) * tmp;
            tmp *= 4294967296.0;
        }
        double r = sum / tmp;
        if (r >= 1.0) r = nextafter(1.0, 0.0);
        u[s] = r;
    }
}

int or_sample(const double* state, int n, const double* u, size_t n_shots,
              uint64_t* out_idx, double* cp_out) {
    const uint64_t dim = 1ull << n;
    double* cp = cp_out ? cp_out : (double*)malloc(dim * sizeof(double));
    if (!cp) return fail(2, "out of host memory");
    /* probabilities x*x + y*y, each product rounded (no contraction) */
    volatile double prod_r, prod_i;
    double sum = 0.0;
    for (uint64_t i = 0; i < dim; ++i) {
        prod_r = state[2 * i] * state[2 * i];
        prod_i = state[2 * i + 1] * state[2 * i + 1];
        cp[i] = prod_r + prod_i;
        sum += cp[i];
    }
    double run = 0.0;
    for (uint64_t i = 0; i < dim; ++i) {
        run += cp[i] / sum;
        cp[i] = run;
    }
    if (dim >= 2) cp[dim - 1] = 1.0;
    for (size_t s = 0; s < n_shots; ++s) {
        if (dim < 2) { out_idx[s] = 0; continue; }
        uint64_t lo = 0, hi = dim;  /* first j with cp[j] >= u */
        while (lo < hi) {
            uint64_t mid = lo + (hi - lo) / 2;
            if (cp[mid] < u[s]) lo = mid + 1; else hi = mid;
        }
        out_idx[s] = lo;
    }
    if (!cp_out) free(cp);
    return 0;
}

/* ---------------------------------------------------------------- adjoint */

static int adjoint_core(const double* psi0, int n, const uint8_t* cmds, size_t nbytes,
                        const int32_t* dep_ptr, const int32_t* dep_param,
                        const double* dep_alpha, int n_params,
                        cplx* phi /* filled by caller after forward when NULL-built */,
                        const uint64_t* xm, const uint64_t* zm, const double* coeff,
                        size_t nt, const double* phi_in, double* grad, double* energy) {
    const uint64_t dim = 1ull << n;
    /* index the records */
    size_t cap = 64, nrec = 0, off = 0;
    rec_t* recs = (rec_t*)malloc(cap * sizeof(rec_t));
    while (off < nbytes) {
        if (nrec == cap) { cap *= 2; recs = (rec_t*)realloc(recs, cap * sizeof(rec_t)); }
        int rc = decode(cmds, nbytes, off, &recs[nrec]);
        if (rc) { free(recs); return rc; }
        int g = recs[nrec].gate;
        if (g == G_RESET || (g == G_MEASURE && recs[nrec].ncb > 0) || (recs[nrec].flags & 1)
                || g == G_BBEGIN) {
            free(recs);
            return fail(2, "trajectory commands (Measure / Reset / classical condition) are not differentiable");
        }
        off += recs[nrec].size;
        ++nrec;
    }
    cplx* psi = (cplx*)calloc(dim, sizeof(cplx));
    cplx* scratch = (cplx*)malloc(dim * sizeof(cplx));
    if (psi0) memcpy(psi, psi0, dim * sizeof(cplx)); else psi[0] = 1.0;
    for (size_t i = 0; i < nrec; ++i) {
        int rc = apply_rec(psi, n, &recs[i]);
        if (rc) { free(recs); free(psi); free(scratch); return rc; }
    }
    if (phi_in) {
        memcpy(phi, phi_in, dim * sizeof(cplx));
    } else {
        or_apply_observable((const double*)psi, (double*)phi, n, xm, zm, coeff, nt);
        if (energy) {
            cplx e = 0;
            for (uint64_t i = 0; i < dim; ++i) e += conj(psi[i]) * phi[i];
            *energy = creal(e);
        }
    }
    for (int p = 0; p < n_params; ++p) grad[p] = 0.0;
    for (size_t idx = nrec; idx-- > 0;) {
        const rec_t* r = &recs[idx];
        if (dep_ptr[idx + 1] > dep_ptr[idx]) {
            memcpy(scratch, psi, dim * sizeof(cplx));
            cplx pref;
            if (!apply_generator(scratch, n, r, &pref)) {
                free(recs); free(psi); free(scratch);
                return fail(3, "run_gradient: gate carries a symbolic parameter but has no adjoint generator rule");
            }
            cplx ip = 0;
            for (uint64_t i = 0; i < dim; ++i) ip += conj(phi[i]) * scratch[i];
            double base = 2.0 * creal(pref * ip);
            for (int d = dep_ptr[idx]; d < dep_ptr[idx + 1]; ++d)
                grad[dep_param[d]] += dep_alpha[d] * base;
        }
        apply_dagger(psi, n, r);
        apply_dagger(phi, n, r);
    }
    free(recs); free(psi); free(scratch);
    return 0;
}

int or_adjoint(const double* psi0, int n, const uint8_t* cmds, size_t nbytes,
               const int32_t* dep_ptr, const int32_t* dep_param, const double* dep_alpha,
               int n_params,
               const uint64_t* xm, const uint64_t* zm, const double* coeff,
               size_t nt, double* grad, double* energy) {
    if (check_terms(n, xm, zm, nt)) return 1;
    cplx* phi = (cplx*)malloc((1ull << n) * sizeof(cplx));
    int rc = adjoint_core(psi0, n, cmds, nbytes, dep_ptr, dep_param, dep_alpha, n_params,
                          phi, xm, zm, coeff, nt, NULL, grad, energy);
    free(phi);
    return rc;
}

int or_adjoint_phi(const double* psi0, int n, const uint8_t* cmds, size_t nbytes,
                   const int32_t* dep_ptr, const int32_t* dep_param, const double* dep_alpha,
                   int n_params, const double* phi_in, double* grad) {
    cplx* phi = (cplx*)malloc((1ull << n) * sizeof(cplx));
    int rc = adjoint_core(psi0, n, cmds, nbytes, dep_ptr, dep_param, dep_alpha, n_params,
                          phi, NULL, NULL, NULL, 0, phi_in, grad, NULL);
    free(phi);
    return rc;
}
