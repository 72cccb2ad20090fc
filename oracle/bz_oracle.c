/* CPU restatement of the reference BZ distance path.  TEST INFRASTRUCTURE ONLY (see
 * bz_oracle.h).  Every function names the reference lines it restates; paths are inside the
 * Quantinuum/Qubitserf tree. */
#include "bz_oracle.h"

#include <stdlib.h>
#include <string.h>

typedef uint64_t u64;

/* ------------------------------------------------------------------ bit-packed matrix
 * Row format of cpp/qsf/bits.hpp:1-63: ceil(cols/64) little-endian words per row. */
typedef struct {
    int rows, cols, stride, cap;
    u64* w;
} mat;

static int words_for(int bits) { return (bits + 63) >> 6; }
static int popc(u64 x) { return __builtin_popcountll(x); }

static mat m_new(int r, int c) {
    mat m;
    m.rows = r; m.cols = c; m.stride = words_for(c); m.cap = r > 0 ? r : 1;
    m.w = (u64*)calloc((size_t)m.cap * (m.stride ? m.stride : 1), sizeof(u64));
    return m;
}
static void m_free(mat* m) { free(m->w); m->w = NULL; m->rows = 0; }
static u64* m_row(const mat* m, int i) { return m->w + (size_t)i * m->stride; }
static mat m_copy(const mat* a) {
    mat m = m_new(a->rows, a->cols);
    if (a->rows) memcpy(m.w, a->w, (size_t)a->rows * a->stride * sizeof(u64));
    return m;
}
static void m_append(mat* m, const u64* src) {
    if (m->rows == m->cap) {
        m->cap *= 2;
        m->w = (u64*)realloc(m->w, (size_t)m->cap * (m->stride ? m->stride : 1) * sizeof(u64));
    }
    memcpy(m_row(m, m->rows), src, (size_t)m->stride * sizeof(u64));
    m->rows++;
}
static int m_get(const mat* m, int i, int j) { return (int)((m_row(m, i)[j >> 6] >> (j & 63)) & 1u); }
static void m_set1(mat* m, int i, int j) { m_row(m, i)[j >> 6] |= 1ull << (j & 63); }
static int v_weight(const u64* v, int s) { int w = 0; for (int i = 0; i < s; ++i) w += popc(v[i]); return w; }
static void v_xor(u64* d, const u64* s, int n) { for (int i = 0; i < n; ++i) d[i] ^= s[i]; }
static int v_dot(const u64* a, const u64* b, int n) {
    u64 acc = 0;
    for (int i = 0; i < n; ++i) acc ^= a[i] & b[i];
    return popc(acc) & 1;
}
static int v_zero(const u64* v, int n) { for (int i = 0; i < n; ++i) if (v[i]) return 0; return 1; }

static mat m_from_dense(const uint8_t* d, int r, int c) {
    mat m = m_new(r, c);
    for (int i = 0; i < r; ++i)
        for (int j = 0; j < c; ++j)
            if (d[(size_t)i * c + j] & 1) m_set1(&m, i, j);
    return m;
}

/* pivot = first row >= rank with a 1, swap, clear the column elsewhere:
 * cpp/qsf/gf2.cpp:25-58 */
static int elim(mat* m, int rank, int col) {
    const int wd = col >> 6;
    const u64 bit = 1ull << (col & 63);
    int sel = -1;
    for (int r = rank; r < m->rows; ++r)
        if (m_row(m, r)[wd] & bit) { sel = r; break; }
    if (sel < 0) return 0;
    if (sel != rank)
        for (int i = 0; i < m->stride; ++i) {
            u64 t = m_row(m, rank)[i];
            m_row(m, rank)[i] = m_row(m, sel)[i];
            m_row(m, sel)[i] = t;
        }
    for (int r = 0; r < m->rows; ++r)
        if (r != rank && (m_row(m, r)[wd] & bit)) v_xor(m_row(m, r), m_row(m, rank), m->stride);
    return 1;
}
static int m_rref(mat* m, int* piv) {
    int rank = 0;
    for (int c = 0; c < m->cols && rank < m->rows; ++c)
        if (elim(m, rank, c)) { if (piv) piv[rank] = c; ++rank; }
    return rank;
}
static int m_rrref(mat* m, const int* cols, int nc, int* piv) {
    int rank = 0;
    for (int i = 0; i < nc && rank < m->rows; ++i)
        if (elim(m, rank, cols[i])) { if (piv) piv[rank] = cols[i]; ++rank; }
    return rank;
}
static void m_drop_zero(mat* m) {
    int out = 0;
    for (int r = 0; r < m->rows; ++r) {
        if (v_zero(m_row(m, r), m->stride)) continue;
        if (out != r) memcpy(m_row(m, out), m_row(m, r), (size_t)m->stride * sizeof(u64));
        ++out;
    }
    m->rows = out;
}
/* cpp/qsf/gf2.cpp:72-94 */
static mat m_nullspace(const mat* in) {
    mat m = m_copy(in);
    int* piv = (int*)malloc(sizeof(int) * (size_t)(m.cols + 1));
    const int rank = m_rref(&m, piv);
    char* isp = (char*)calloc((size_t)m.cols + 1, 1);
    for (int i = 0; i < rank; ++i) isp[piv[i]] = 1;
    mat ns = m_new(m.cols - rank, m.cols);
    int out = 0;
    for (int f = 0; f < m.cols; ++f) {
        if (isp[f]) continue;
        m_set1(&ns, out, f);
        for (int r = 0; r < rank; ++r)
            if (m_get(&m, r, f)) m_set1(&ns, out, piv[r]);
        ++out;
    }
    free(piv); free(isp); m_free(&m);
    return ns;
}
static mat m_transpose(const mat* m) {
    mat t = m_new(m->cols, m->rows);
    for (int i = 0; i < m->rows; ++i)
        for (int j = 0; j < m->cols; ++j)
            if (m_get(m, i, j)) m_set1(&t, j, i);
    return t;
}
static int in_rowspace_packed(const mat* G, const u64* v) {
    mat R = m_copy(G);
    int* piv = (int*)malloc(sizeof(int) * (size_t)(R.cols + 1));
    const int rank = m_rref(&R, piv);
    u64* t = (u64*)malloc(sizeof(u64) * (size_t)(R.stride + 1));
    memcpy(t, v, (size_t)R.stride * sizeof(u64));
    for (int r = 0; r < rank; ++r)
        if ((t[piv[r] >> 6] >> (piv[r] & 63)) & 1u) v_xor(t, m_row(&R, r), R.stride);
    const int z = v_zero(t, R.stride);
    free(t); free(piv); m_free(&R);
    return z;
}
static u64* pack_vec(const uint8_t* v, int n) {
    u64* o = (u64*)calloc((size_t)words_for(n) + 1, sizeof(u64));
    for (int j = 0; j < n; ++j)
        if (v[j] & 1) o[j >> 6] |= 1ull << (j & 63);
    return o;
}

/* ------------------------------------------------------------------ problems
 * DistProblem of cpp/distfind/css.hpp:21-30 */
typedef struct {
    int n;
    mat gen, check;
    int even, count_all, seed_upper;
    int symplectic, qubits;
} problem;

static void p_free(problem* p) { m_free(&p->gen); m_free(&p->check); }

static int lowest_set(const u64* v, int s) {
    for (int i = 0; i < s; ++i)
        if (v[i]) return i * 64 + __builtin_ctzll(v[i]);
    return -1;
}
/* reducing basis, cpp/distfind/css.cpp:98-126 */
typedef struct { mat rows; int* piv; } reducer;
static int red_reduce(const reducer* b, u64* v) {
    for (int i = 0; i < b->rows.rows; ++i) {
        const int p = b->piv[i];
        if ((v[p >> 6] >> (p & 63)) & 1u) v_xor(v, m_row(&b->rows, i), b->rows.stride);
    }
    return !v_zero(v, b->rows.stride);
}
static void red_add(reducer* b, const u64* v) {
    m_append(&b->rows, v);
    b->piv = (int*)realloc(b->piv, sizeof(int) * (size_t)b->rows.rows);
    b->piv[b->rows.rows - 1] = lowest_set(v, b->rows.stride);
}
/* cpp/distfind/css.cpp:175-186 */
static mat quotient_basis(const mat* self, const mat* other) {
    mat ko = m_nullspace(other);
    reducer b;
    b.rows = m_new(0, self->cols);
    b.piv = NULL;
    u64* t = (u64*)malloc(sizeof(u64) * (size_t)(self->stride + 1));
    for (int i = 0; i < self->rows; ++i) {
        memcpy(t, m_row(self, i), (size_t)self->stride * sizeof(u64));
        if (red_reduce(&b, t)) red_add(&b, t);
    }
    mat out = m_new(0, self->cols);
    for (int i = 0; i < ko.rows; ++i) {
        memcpy(t, m_row(&ko, i), (size_t)ko.stride * sizeof(u64));
        if (!red_reduce(&b, t)) continue;
        red_add(&b, t);
        m_append(&out, m_row(&ko, i));
    }
    free(t); free(b.piv); m_free(&b.rows); m_free(&ko);
    return out;
}
static int all_even(const mat* m) {
    for (int i = 0; i < m->rows; ++i) if (v_weight(m_row(m, i), m->stride) & 1) return 0;
    return 1;
}
static int min_row_weight(const mat* m) {
    int b = 1 << 30;
    for (int i = 0; i < m->rows; ++i) {
        const int w = v_weight(m_row(m, i), m->stride);
        if (w < b) b = w;
    }
    return b;
}
/* cpp/distfind/css.cpp:159-168 */
static problem build(const mat* self, const mat* other) {
    problem p;
    memset(&p, 0, sizeof(p));
    p.n = self->cols;
    p.gen = m_nullspace(self);
    p.check = quotient_basis(self, other);
    mat logi = quotient_basis(other, self);
    p.even = all_even(&p.gen);
    p.seed_upper = logi.rows ? min_row_weight(&logi) : 0;
    m_free(&logi);
    return p;
}
static problem classical_problem(const mat* H) {  /* cpp/distfind/css.cpp:192-201 */
    problem p;
    memset(&p, 0, sizeof(p));
    p.n = H->cols;
    p.gen = m_nullspace(H);
    p.check = m_new(0, H->cols);
    p.count_all = 1;
    p.even = all_even(&p.gen);
    p.seed_upper = p.gen.rows ? min_row_weight(&p.gen) : 0;
    return p;
}
static mat gram(const mat* A, const mat* B) {
    mat E = m_new(A->rows, B->rows);
    for (int i = 0; i < A->rows; ++i)
        for (int j = 0; j < B->rows; ++j)
            if (v_dot(m_row(A, i), m_row(B, j), A->stride)) m_set1(&E, i, j);
    return E;
}
static mat combine(const mat* C, const mat* B) {
    mat o = m_new(C->rows, B->cols);
    for (int i = 0; i < C->rows; ++i)
        for (int j = 0; j < B->rows; ++j)
            if (m_get(C, i, j)) v_xor(m_row(&o, i), m_row(B, j), B->stride);
    return o;
}
/* cpp/distfind/css.cpp:203-220 */
static problem subsystem_problem(const mat* Gx, const mat* Gz, char which) {
    mat E = gram(Gx, Gz), Et = m_transpose(&E);
    mat n1 = m_nullspace(&Et), n2 = m_nullspace(&E);
    mat Sx = combine(&n1, Gx), Sz = combine(&n2, Gz);
    m_rref(&Sx, NULL); m_drop_zero(&Sx);
    m_rref(&Sz, NULL); m_drop_zero(&Sz);
    problem p = which == 'X' ? build(&Sz, Gx) : build(&Sx, Gz);
    m_free(&E); m_free(&Et); m_free(&n1); m_free(&n2); m_free(&Sx); m_free(&Sz);
    return p;
}
/* cpp/distfind/css.cpp:231-255 */
static problem coset_problem(const mat* G, const u64* v) {
    problem p;
    memset(&p, 0, sizeof(p));
    const int n = G->cols;
    p.n = n;
    mat M = m_copy(G);
    m_append(&M, v);
    m_rref(&M, NULL);
    m_drop_zero(&M);
    p.gen = M;
    mat N = m_nullspace(G);
    p.check = m_new(0, n);
    for (int i = 0; i < N.rows; ++i)
        if (v_dot(m_row(&N, i), v, N.stride)) { m_append(&p.check, m_row(&N, i)); break; }
    m_free(&N);
    p.even = all_even(&p.gen);
    p.seed_upper = v_weight(v, words_for(n));
    return p;
}
/* cpp/distfind/stab.cpp:13-178 */
static mat sw_swap(const mat* m) {
    const int q = m->cols / 2;
    mat o = m_new(m->rows, m->cols);
    for (int i = 0; i < m->rows; ++i)
        for (int j = 0; j < q; ++j) {
            if (m_get(m, i, j)) m_set1(&o, i, q + j);
            if (m_get(m, i, q + j)) m_set1(&o, i, j);
        }
    return o;
}
static int sw_weight(const u64* r, int q) {
    int w = 0;
    for (int j = 0; j < q; ++j) {
        const int z = (int)((r[j >> 6] >> (j & 63)) & 1u);
        const int x = (int)((r[(q + j) >> 6] >> ((q + j) & 63)) & 1u);
        w += z | x;
    }
    return w;
}
static int is_css(const mat* S) {
    const int q = S->cols / 2;
    for (int i = 0; i < S->rows; ++i) {
        int hz = 0, hx = 0;
        for (int j = 0; j < q; ++j) { hz |= m_get(S, i, j); hx |= m_get(S, i, q + j); }
        if (hz && hx) return 0;
    }
    return 1;
}
static void split_css(const mat* S, mat* Hx, mat* Hz) {
    const int q = S->cols / 2;
    *Hx = m_new(0, q);
    *Hz = m_new(0, q);
    mat zr = m_new(1, q), xr = m_new(1, q);
    for (int i = 0; i < S->rows; ++i) {
        memset(zr.w, 0, (size_t)zr.stride * 8);
        memset(xr.w, 0, (size_t)xr.stride * 8);
        int hz = 0, hx = 0;
        for (int j = 0; j < q; ++j) {
            if (m_get(S, i, j)) { m_set1(&zr, 0, j); hz = 1; }
            if (m_get(S, i, q + j)) { m_set1(&xr, 0, j); hx = 1; }
        }
        if (hx) m_append(Hx, xr.w);
        else if (hz) m_append(Hz, zr.w);
    }
    m_free(&zr); m_free(&xr);
}
static mat sympl_center(const mat* G) {
    mat s = sw_swap(G), gr = gram(G, &s), ns = m_nullspace(&gr);
    mat C = combine(&ns, G);
    m_rref(&C, NULL);
    m_drop_zero(&C);
    m_free(&s); m_free(&gr); m_free(&ns);
    return C;
}
static problem sympl_problem(const mat* Sn, const mat* Gt) {
    problem p;
    memset(&p, 0, sizeof(p));
    p.symplectic = 1;
    p.n = Sn->cols;
    p.qubits = Sn->cols / 2;
    mat s1 = sw_swap(Sn);
    p.gen = m_nullspace(&s1);
    mat s2 = sw_swap(Gt);
    mat L = quotient_basis(Sn, &s2);
    p.check = sw_swap(&L);
    int best = 0;
    for (int i = 0; i < p.gen.rows; ++i) {
        if (in_rowspace_packed(Gt, m_row(&p.gen, i))) continue;
        const int w = sw_weight(m_row(&p.gen, i), p.qubits);
        if (best == 0 || w < best) best = w;
    }
    p.seed_upper = best;
    m_free(&s1); m_free(&s2); m_free(&L);
    return p;
}
static problem isometry(const problem* sp) {
    const int q = sp->qubits;
    problem e;
    memset(&e, 0, sizeof(e));
    e.n = 3 * q;
    e.even = 1;
    e.count_all = sp->count_all;
    e.seed_upper = sp->seed_upper > 0 ? 2 * sp->seed_upper : 0;
    e.gen = m_new(sp->gen.rows, e.n);
    for (int i = 0; i < sp->gen.rows; ++i)
        for (int j = 0; j < q; ++j) {
            const int a = m_get(&sp->gen, i, j), b = m_get(&sp->gen, i, q + j);
            if (a) m_set1(&e.gen, i, j);
            if (b) m_set1(&e.gen, i, q + j);
            if (a ^ b) m_set1(&e.gen, i, 2 * q + j);
        }
    e.check = m_new(sp->check.rows, e.n);
    for (int i = 0; i < sp->check.rows; ++i)
        for (int j = 0; j < sp->n; ++j)
            if (m_get(&sp->check, i, j)) m_set1(&e.check, i, j);
    return e;
}

/* ------------------------------------------------------------------ information sets
 * cpp/distfind/css.cpp:177-366 */
typedef struct { mat g; int rank; } gset;
typedef struct { gset* s; int n, cap; } gseq;

static void gs_push(gseq* q, mat g, int rank) {
    if (q->n == q->cap) {
        q->cap = q->cap ? 2 * q->cap : 4;
        q->s = (gset*)realloc(q->s, sizeof(gset) * (size_t)q->cap);
    }
    q->s[q->n].g = g;
    q->s[q->n].rank = rank;
    q->n++;
}
static void gs_free(gseq* q) {
    for (int i = 0; i < q->n; ++i) m_free(&q->s[i].g);
    free(q->s);
    q->s = NULL; q->n = q->cap = 0;
}
static gseq greedy(const mat* gen) {
    gseq q = {0};
    const int n = gen->cols;
    int* active = (int*)malloc(sizeof(int) * (size_t)(n + 1));
    int* next = (int*)malloc(sizeof(int) * (size_t)(n + 1));
    int* piv = (int*)malloc(sizeof(int) * (size_t)(n + 1));
    char* isp = (char*)malloc((size_t)n + 1);
    char* nz = (char*)malloc((size_t)n + 1);
    int na = n;
    for (int i = 0; i < n; ++i) active[i] = i;
    mat work = m_copy(gen);
    while (na > 0) {
        const int np = m_rrref(&work, active, na, piv);
        gs_push(&q, m_copy(&work), np);
        memset(isp, 0, (size_t)n + 1);
        memset(nz, 0, (size_t)n + 1);
        for (int i = 0; i < np; ++i) isp[piv[i]] = 1;
        for (int r = 0; r < work.rows; ++r)
            for (int i = 0; i < na; ++i)
                if (m_get(&work, r, active[i])) nz[active[i]] = 1;
        int nn = 0;
        for (int i = 0; i < na; ++i)
            if (!isp[active[i]] && nz[active[i]]) next[nn++] = active[i];
        if (nn == na) break;
        memcpy(active, next, sizeof(int) * (size_t)nn);
        na = nn;
    }
    m_free(&work);
    free(active); free(next); free(piv); free(isp); free(nz);
    return q;
}

/* matroid partition by augmenting DFS, cpp/distfind/css.cpp:274-328 */
typedef struct { int* v; int n, cap; } ivec;
static void iv_push(ivec* a, int x) {
    if (a->n == a->cap) { a->cap = a->cap ? 2 * a->cap : 8; a->v = (int*)realloc(a->v, sizeof(int) * (size_t)a->cap); }
    a->v[a->n++] = x;
}
static void iv_erase(ivec* a, int x) {
    for (int i = 0; i < a->n; ++i)
        if (a->v[i] == x) { memmove(a->v + i, a->v + i + 1, sizeof(int) * (size_t)(a->n - i - 1)); a->n--; return; }
}
/* sorted symmetric difference */
static ivec symdiff(const ivec* a, const ivec* b) {
    ivec r = {0};
    int i = 0, j = 0;
    while (i < a->n && j < b->n) {
        if (a->v[i] < b->v[j]) iv_push(&r, a->v[i++]);
        else if (b->v[j] < a->v[i]) iv_push(&r, b->v[j++]);
        else { ++i; ++j; }
    }
    while (i < a->n) iv_push(&r, a->v[i++]);
    while (j < b->n) iv_push(&r, b->v[j++]);
    return r;
}
typedef struct {
    const u64* col; int kw; int n;
    ivec* cls; int ncls, capcls;
    char* visited;
} mpart;

/* express z over class c: returns in_span, fills circuit (sorted) */
static int express(const mpart* P, const ivec* cls, int z, ivec* circuit) {
    const int kw = P->kw;
    int nb = 0;
    u64* basis = (u64*)malloc(sizeof(u64) * (size_t)(cls->n + 1) * (size_t)kw);
    int* bp = (int*)malloc(sizeof(int) * (size_t)(cls->n + 1));
    ivec* bo = (ivec*)calloc((size_t)cls->n + 1, sizeof(ivec));
    u64* v = (u64*)malloc(sizeof(u64) * (size_t)kw);
    for (int t = 0; t < cls->n; ++t) {
        const int idx = cls->v[t];
        memcpy(v, P->col + (size_t)idx * kw, sizeof(u64) * (size_t)kw);
        ivec orig = {0};
        iv_push(&orig, idx);
        for (int b = 0; b < nb; ++b) {
            const int p = bp[b];
            if ((v[p >> 6] >> (p & 63)) & 1u) {
                v_xor(v, basis + (size_t)b * kw, kw);
                ivec s = symdiff(&orig, &bo[b]);
                free(orig.v);
                orig = s;
            }
        }
        const int lb = lowest_set(v, kw);
        if (lb >= 0) {
            memcpy(basis + (size_t)nb * kw, v, sizeof(u64) * (size_t)kw);
            bp[nb] = lb;
            bo[nb] = orig;
            ++nb;
        } else {
            free(orig.v);
        }
    }
    memcpy(v, P->col + (size_t)z * kw, sizeof(u64) * (size_t)kw);
    ivec orig = {0};
    for (int b = 0; b < nb; ++b) {
        const int p = bp[b];
        if ((v[p >> 6] >> (p & 63)) & 1u) {
            v_xor(v, basis + (size_t)b * kw, kw);
            ivec s = symdiff(&orig, &bo[b]);
            free(orig.v);
            orig = s;
        }
    }
    const int zero = v_zero(v, kw);
    if (circuit) {
        circuit->n = 0;
        if (zero) for (int i = 0; i < orig.n; ++i) iv_push(circuit, orig.v[i]);
    }
    free(orig.v);
    for (int b = 0; b < nb; ++b) free(bo[b].v);
    free(bo); free(bp); free(basis); free(v);
    return zero;
}
static int place(mpart* P, int z, int forbidden) {
    for (int c = 0; c < P->ncls; ++c) {
        if (c == forbidden) continue;
        if (!express(P, &P->cls[c], z, NULL)) { iv_push(&P->cls[c], z); return 1; }
    }
    for (int c = 0; c < P->ncls; ++c) {
        if (c == forbidden) continue;
        ivec circ = {0};
        if (!express(P, &P->cls[c], z, &circ)) { free(circ.v); continue; }
        for (int i = 0; i < circ.n; ++i) {
            const int y = circ.v[i];
            if (P->visited[y]) continue;
            P->visited[y] = 1;
            iv_erase(&P->cls[c], y);
            iv_push(&P->cls[c], z);
            if (place(P, y, c)) { free(circ.v); return 1; }
            iv_erase(&P->cls[c], z);
            iv_push(&P->cls[c], y);
        }
        free(circ.v);
    }
    return 0;
}
static int count_full(const gseq* q, int K) {
    int f = 0;
    for (int i = 0; i < q->n; ++i) f += q->s[i].rank == K;
    return f;
}
static gseq gamma_sequence(const mat* gen) {
    const int K = gen->rows, n = gen->cols;
    gseq gr = greedy(gen);
    if (K == 0) return gr;
    int nnz = 0;
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < K; ++i)
            if (m_get(gen, i, j)) { ++nnz; break; }
    const int max_full = nnz / K, gfull = count_full(&gr, K);
    if (gfull >= max_full || n > 200) return gr;
    mpart P;
    memset(&P, 0, sizeof(P));
    P.kw = words_for(K);
    P.n = n;
    u64* col = (u64*)calloc((size_t)n * P.kw + 1, sizeof(u64));
    ivec nonzero = {0}, zeros = {0};
    for (int j = 0; j < n; ++j) {
        int nzc = 0;
        for (int i = 0; i < K; ++i)
            if (m_get(gen, i, j)) { col[(size_t)j * P.kw + (i >> 6)] |= 1ull << (i & 63); nzc = 1; }
        iv_push(nzc ? &nonzero : &zeros, j);
    }
    P.col = col;
    P.visited = (char*)calloc((size_t)n + 1, 1);
    P.capcls = n + 1;
    P.cls = (ivec*)calloc((size_t)P.capcls, sizeof(ivec));
    for (int t = 0; t < nonzero.n; ++t) {
        memset(P.visited, 0, (size_t)n + 1);
        if (!place(&P, nonzero.v[t], -1)) iv_push(&P.cls[P.ncls++], nonzero.v[t]);
    }
    if (P.ncls == 0) P.ncls = 1;
    for (int t = 0; t < zeros.n; ++t) iv_push(&P.cls[0], zeros.v[t]);
    /* classes by size, descending (stable here; the reference's std::sort may order
       equal-size classes differently, which never changes the rank multiset) */
    int* ord = (int*)malloc(sizeof(int) * (size_t)P.ncls);
    for (int i = 0; i < P.ncls; ++i) ord[i] = i;
    for (int i = 1; i < P.ncls; ++i) {
        const int x = ord[i];
        int j = i - 1;
        while (j >= 0 && P.cls[ord[j]].n < P.cls[x].n) { ord[j + 1] = ord[j]; --j; }
        ord[j + 1] = x;
    }
    gseq seq = {0};
    int* piv = (int*)malloc(sizeof(int) * (size_t)(n + 1));
    for (int i = 0; i < P.ncls; ++i) {
        const ivec* c = &P.cls[ord[i]];
        if (c->n == 0) continue;
        mat w = m_copy(gen);
        const int np = m_rrref(&w, c->v, c->n, piv);
        gs_push(&seq, w, np);
    }
    free(piv); free(ord);
    for (int i = 0; i < P.capcls; ++i) free(P.cls[i].v);
    free(P.cls); free(P.visited); free(col); free(nonzero.v); free(zeros.v);
    if (seq.n == 0 || count_full(&seq, K) <= gfull) { gs_free(&seq); return gr; }
    gs_free(&gr);
    return seq;
}
/* stable sort by rank, descending (cpp/distfind/bz.cpp:141-143) */
static void sort_by_rank(gseq* q) {
    for (int i = 1; i < q->n; ++i) {
        gset x = q->s[i];
        int j = i - 1;
        while (j >= 0 && q->s[j].rank < x.rank) { q->s[j + 1] = q->s[j]; --j; }
        q->s[j + 1] = x;
    }
}

/* ------------------------------------------------------------------ enumeration */
static int logical_of(const u64* cw, int kcheck, const u64* check, int stride) {
    if (kcheck == 0) return 1;
    for (int c = 0; c < kcheck; ++c)
        if (v_dot(check + (size_t)c * stride, cw, stride)) return 1;
    return 0;
}

int orc_enumerate(int n, int stride, int K, int d, int ng, const uint64_t* gamma, int kcheck,
                  const uint64_t* check, int current_best, unsigned long long* counts,
                  int* arg_g, unsigned long long* arg_rank) {
    (void)n;
    int* pos = (int*)malloc(sizeof(int) * (size_t)(d + 1));
    u64* cw = (u64*)malloc(sizeof(u64) * (size_t)(stride + 1));
    for (int i = 0; i < d; ++i) pos[i] = i;
    int best = current_best, bg = -1;
    u64 brank = ~0ull, rank = 0;
    for (int g = 0; g < ng; ++g) if (counts) counts[g] = 0;
    for (;;) {
        for (int g = 0; g < ng; ++g) {
            const u64* G = gamma + (size_t)g * K * stride;
            memset(cw, 0, sizeof(u64) * (size_t)stride);
            for (int i = 0; i < d; ++i) v_xor(cw, G + (size_t)pos[i] * stride, stride);
            if (counts) counts[g]++;
            if (!logical_of(cw, kcheck, check, stride)) continue;
            const int w = v_weight(cw, stride);
            if (w >= current_best) continue;
            if (w < best || (w == best && (g < bg || (g == bg && rank < brank)))) {
                best = w; bg = g; brank = rank;
            }
        }
        int j = d - 1;
        while (j >= 0 && pos[j] == K - d + j) --j;
        if (j < 0) break;
        ++pos[j];
        for (int t = j + 1; t < d; ++t) pos[t] = pos[t - 1] + 1;
        ++rank;
    }
    if (arg_g) *arg_g = bg;
    if (arg_rank) *arg_rank = brank;
    free(pos); free(cw);
    return best;
}

/* cpp/qsf/enum_core.hpp:109-194: outer d-1 positions with a running XOR base, inner sweep
 * of the last position with a per-word early exit against the bound. */
static int enum_level(int stride, int K, int d, int ng, const u64* gamma, int kcheck,
                      const u64* check, int bound) {
    const int M = d - 1;
    int* pos = (int*)malloc(sizeof(int) * (size_t)(d + 1));
    u64* cw = (u64*)malloc(sizeof(u64) * (size_t)(stride + 1));
    u64* c2 = (u64*)malloc(sizeof(u64) * (size_t)(stride + 1));
    for (int g = 0; g < ng; ++g) {
        const u64* G = gamma + (size_t)g * K * stride;
        for (int i = 0; i < M; ++i) pos[i] = i;
        memset(cw, 0, sizeof(u64) * (size_t)stride);
        for (int i = 0; i < M; ++i) v_xor(cw, G + (size_t)pos[i] * stride, stride);
        for (;;) {
            const int start = M ? pos[M - 1] + 1 : 0;
            for (int r = start; r < K; ++r) {
                const u64* row = G + (size_t)r * stride;
                int wt = 0, light = 1;
                for (int w = 0; w < stride && light; ++w) {
                    wt += popc(cw[w] ^ row[w]);
                    light = wt < bound;
                }
                if (!light) continue;
                for (int w = 0; w < stride; ++w) c2[w] = cw[w] ^ row[w];
                if (logical_of(c2, kcheck, check, stride)) bound = wt;
            }
            if (M == 0) break;
            /* next outer (M-subset of [0, K-1)) */
            int j = M - 1;
            while (j >= 0 && pos[j] == (K - 1) - M + j) --j;
            if (j < 0) break;
            for (int t = j; t < M; ++t) v_xor(cw, G + (size_t)pos[t] * stride, stride);
            ++pos[j];
            for (int t = j + 1; t < M; ++t) pos[t] = pos[t - 1] + 1;
            for (int t = j; t < M; ++t) v_xor(cw, G + (size_t)pos[t] * stride, stride);
        }
    }
    free(pos); free(cw); free(c2);
    return bound;
}

int orc_enumerate_fast(int n, int stride, int K, int d, int ng, const uint64_t* gamma,
                       int kcheck, const uint64_t* check, int current_best) {
    (void)n;
    if (d < 1 || d > K) return current_best;
    return enum_level(stride, K, d, ng, gamma, kcheck, check, current_best);
}

/* ------------------------------------------------------------------ BZ schedule
 * cpp/distfind/bz.cpp:72-370 */
typedef struct {
    int has, K, ng, stride, kcheck, even, maxw;
    int* ranks;
    u64* gamma;
    u64* check;
    int inner, outer, level, proven, resolved;
} side;

static u64 splitmix(u64* s) {
    u64 z = (*s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

/* random information sets (any logical row bounds the distance; bz.cpp:60-69) */
static int seed_trials(const problem* p, int best, int trials) {
    const int n = p->n;
    int* cols = (int*)malloc(sizeof(int) * (size_t)(n + 1));
    u64 st = 0x5eedull;
    for (int t = 0; t < trials; ++t) {
        for (int i = 0; i < n; ++i) cols[i] = i;
        for (int i = n - 1; i > 0; --i) {
            const int j = (int)(splitmix(&st) % (u64)(i + 1));
            const int x = cols[i]; cols[i] = cols[j]; cols[j] = x;
        }
        mat M = m_copy(&p->gen);
        m_rrref(&M, cols, n, NULL);
        for (int r = 0; r < M.rows; ++r) {
            const int w = v_weight(m_row(&M, r), M.stride);
            if (w == 0 || w >= best) continue;
            int logical = p->count_all;
            for (int c = 0; c < p->check.rows && !logical; ++c)
                if (v_dot(m_row(&p->check, c), m_row(&M, r), M.stride)) logical = 1;
            if (logical) best = w;
        }
        m_free(&M);
    }
    free(cols);
    return best;
}

static void side_setup(side* S, const problem* p, const orc_options* opt) {
    memset(S, 0, sizeof(*S));
    S->K = p->gen.rows;
    S->even = p->even;
    S->has = !(S->K == 0 || (!p->count_all && p->check.rows == 0));
    if (!S->has) { S->resolved = 1; return; }
    gseq q = gamma_sequence(&p->gen);
    sort_by_rank(&q);
    S->ng = q.n;
    S->stride = words_for(p->n);
    S->ranks = (int*)malloc(sizeof(int) * (size_t)q.n);
    S->gamma = (u64*)calloc((size_t)q.n * S->K * S->stride + 1, sizeof(u64));
    for (int g = 0; g < q.n; ++g) {
        S->ranks[g] = q.s[g].rank;
        memcpy(S->gamma + (size_t)g * S->K * S->stride, q.s[g].g.w,
               sizeof(u64) * (size_t)S->K * S->stride);
    }
    gs_free(&q);
    S->kcheck = p->count_all ? 0 : p->check.rows;
    S->check = (u64*)calloc((size_t)S->kcheck * S->stride + 1, sizeof(u64));
    if (S->kcheck) memcpy(S->check, p->check.w, sizeof(u64) * (size_t)S->kcheck * S->stride);
    S->inner = p->seed_upper > 0 ? p->seed_upper : ORC_WEIGHT_NONE;
    if (opt && opt->seed_trials > 0) S->inner = seed_trials(p, S->inner, opt->seed_trials);
    S->maxw = S->K;
}
static void side_free(side* S) { free(S->ranks); free(S->gamma); free(S->check); }

static int outer_at(const side* S, int w) {
    int o = 0;
    for (int g = 0; g < S->ng; ++g) {
        const int t = (w + 1) - (S->K - S->ranks[g]);
        if (t > 0) o += t;
    }
    if (S->even) o += o & 1;
    return o;
}
/* saturating C(n,k) for level counts */
static unsigned long long binom_simple(int n, int k) {
    if (k < 0 || k > n) return 0;
    if (k > n - k) k = n - k;
    unsigned long long r = 1;
    for (int i = 1; i <= k; ++i) {
        const unsigned __int128 t = (unsigned __int128)r * (unsigned)(n - k + i) / (unsigned)i;
        if (t > ~0ull) return ~0ull;
        r = (unsigned long long)t;
    }
    return r;
}

static int active_at(const side* S, int w) {
    int a = 0;
    while (a < S->ng && (w + 1) - (S->K - S->ranks[a]) > 0) ++a;
    return a;
}

typedef struct { const orc_options* opt; int n; orc_result* r; } recorder;
static void record_level(recorder* R, int side_idx, int w, int active, int K) {
    R->r->codewords += binom_simple(K, w) * (unsigned long long)active;
    const orc_options* o = R->opt;
    if (!o || !o->levels_w || R->n >= o->cap) return;
    o->levels_w[R->n] = w;
    if (o->levels_active) o->levels_active[R->n] = active;
    if (o->levels_side) o->levels_side[R->n] = side_idx;
    R->n++;
}

/* one level of a side (cpp/distfind/bz.cpp:257-271) */
static void side_step(side* S, int w, recorder* R, int side_idx) {
    const int active = active_at(S, w);
    record_level(R, side_idx, w, active, S->K);
    int found = ORC_WEIGHT_NONE;
    if (active > 0)
        found = enum_level(S->stride, S->K, w, active, S->gamma, S->kcheck, S->check, S->inner);
    if (found < S->inner) S->inner = found;
    S->level++;
    S->outer = outer_at(S, w);
}

/* bz_distance, cpp/distfind/bz.cpp:118-228 */
static void bz_single(const problem* p, const orc_options* opt, orc_result* r) {
    memset(r, 0, sizeof(*r));
    recorder R = {opt, 0, r};
    side S;
    side_setup(&S, p, opt);
    if (!S.has) { r->distance = -1; side_free(&S); return; }
    const int nostop = opt && opt->no_early_stop;
    for (int w = 1; w <= S.maxw; ++w) {
        side_step(&S, w, &R, 0);
        if (S.inner <= S.outer && !nostop) { S.proven = 1; break; }
    }
    r->distance = S.inner >= ORC_WEIGHT_NONE ? -1 : S.inner;
    r->levels = S.level;
    r->lower_bound = S.outer;
    r->proven = S.proven;
    side_free(&S);
}

/* bz_min_interleaved, cpp/distfind/bz.cpp:296-357 (cap_to_min) */
static void bz_min(const problem* pz, const problem* px, const orc_options* opt,
                   orc_result* r) {
    memset(r, 0, sizeof(*r));
    recorder R = {opt, 0, r};
    side Z, X;
    side_setup(&Z, pz, opt);
    side_setup(&X, px, opt);
    side* sides[2] = {&Z, &X};
    int best = ORC_WEIGHT_NONE;
    if (Z.has && Z.inner < best) best = Z.inner;
    if (X.has && X.inner < best) best = X.inner;
    const int mz = Z.has ? Z.maxw : 0, mx = X.has ? X.maxw : 0;
    const int maxw = mz > mx ? mz : mx;
    for (int w = 1; w <= maxw; ++w) {
        for (int si = 0; si < 2; ++si) {
            side* S = sides[si];
            if (S->resolved || w > S->maxw) continue;
            if (S->outer >= best) { S->resolved = 1; continue; }
            side_step(S, w, &R, si);
            if (S->inner < best) best = S->inner;
            if (S->inner <= S->outer) { S->proven = 1; S->resolved = 1; }
            else if (S->outer >= best) S->resolved = 1;
        }
        if (Z.resolved && X.resolved) break;
    }
    const int vz = Z.has ? Z.inner : ORC_WEIGHT_NONE, vx = X.has ? X.inner : ORC_WEIGHT_NONE;
    const int dist = vz < vx ? vz : vx;
    r->distance = dist >= ORC_WEIGHT_NONE ? -1 : dist;
    const int lz = Z.has ? Z.outer : ORC_WEIGHT_NONE, lx = X.has ? X.outer : ORC_WEIGHT_NONE;
    const int lb = lz < lx ? lz : lx;
    r->lower_bound = lb >= ORC_WEIGHT_NONE ? 0 : lb;
    r->levels = Z.level > X.level ? Z.level : X.level;
    r->proven = Z.resolved && X.resolved && dist < ORC_WEIGHT_NONE;
    side_free(&Z);
    side_free(&X);
}


/* ------------------------------------------------------------------ meet in the middle
 * method "mitm", cpp/distfind/mitm.cpp:1-552: with H = nullspace(code_gen), level d hits when
 * a left part (coordinates [0, nL)) and a right part ([nL, ncoord)) of weights wL + wR = d
 * share their syndrome (XOR of H's columns) and, unless every codeword counts, differ in
 * their logical fingerprint (XOR of the detector's columns).  Symplectic problems split
 * qubits and give each chosen qubit Z, X or Y (enumerate_side_sym, mitm.cpp:158-199).  The
 * reference joins with a hash map; this restatement sorts the left parts by (syndrome,
 * fingerprint) and binary-searches every right part. */
typedef struct {
    int sw, lw, kw;          /* u64 words: syndrome, fingerprint, record */
    int ncoord, nL, qubits, sym, count_all;
    u64* cols;               /* ncols x kw: syndrome then fingerprint of each column */
} mitm_view;

static int mitm_kw;
static int cmp_rec(const void* a, const void* b) {
    const u64* x = (const u64*)a;
    const u64* y = (const u64*)b;
    for (int i = 0; i < mitm_kw; ++i)
        if (x[i] != y[i]) return x[i] < y[i] ? -1 : 1;
    return 0;
}

static mitm_view mitm_view_of(const problem* p) {
    mitm_view v;
    mat H = m_nullspace(&p->gen);
    v.sym = p->symplectic;
    v.qubits = p->qubits;
    v.count_all = p->count_all;
    v.ncoord = v.sym ? p->qubits : p->n;
    v.nL = v.ncoord / 2;
    v.sw = words_for(H.rows);
    v.lw = v.count_all ? 0 : words_for(p->check.rows);
    v.kw = v.sw + v.lw;
    if (v.kw == 0) v.kw = 1;   /* a record of one zero word */
    v.cols = (u64*)calloc((size_t)p->n * v.kw + 1, sizeof(u64));
    for (int j = 0; j < p->n; ++j) {
        u64* c = v.cols + (size_t)j * v.kw;
        for (int i = 0; i < H.rows; ++i)
            if (m_get(&H, i, j)) c[i >> 6] |= 1ull << (i & 63);
        if (!v.count_all)
            for (int i = 0; i < p->check.rows; ++i)
                if (m_get(&p->check, i, j)) c[v.sw + (i >> 6)] |= 1ull << (i & 63);
    }
    m_free(&H);
    return v;
}

/* every part of weight w over coordinates [first, first + m): records of kw words */
static u64* mitm_parts(const mitm_view* v, int first, int m, int w, size_t* count) {
    size_t n = 1;
    for (int i = 1; i <= w; ++i) n = n * (size_t)(m - w + i) / (size_t)i;
    size_t p3 = 1;
    if (v->sym)
        for (int i = 0; i < w; ++i) p3 *= 3;
    *count = n * p3;
    u64* out = (u64*)calloc(*count * v->kw + 1, sizeof(u64));
    int* pos = (int*)malloc(sizeof(int) * (size_t)(w + 1));
    int* pa = (int*)calloc((size_t)w + 1, sizeof(int));
    for (int i = 0; i < w; ++i) pos[i] = i;
    size_t k = 0;
    for (;;) {
        for (size_t q = 0; q < p3; ++q) {
            /* base-3 odometer value q: digit i picks Z (0), X (1) or Y (2) on qubit pos[i] */
            size_t t = q;
            for (int i = 0; i < w; ++i) { pa[i] = (int)(t % 3); t /= 3; }
            u64* r = out + k * v->kw;
            for (int i = 0; i < w; ++i) {
                const int coord = first + pos[i];
                if (!v->sym) {
                    v_xor(r, v->cols + (size_t)coord * v->kw, v->kw);
                } else {
                    if (pa[i] != 1) v_xor(r, v->cols + (size_t)coord * v->kw, v->kw);
                    if (pa[i] != 0) v_xor(r, v->cols + (size_t)(v->qubits + coord) * v->kw, v->kw);
                }
            }
            ++k;
        }
        int j = w - 1;
        while (j >= 0 && pos[j] == m - w + j) --j;
        if (j < 0) break;
        ++pos[j];
        for (int t2 = j + 1; t2 < w; ++t2) pos[t2] = pos[t2 - 1] + 1;
    }
    free(pos);
    free(pa);
    return out;
}

/* has_codeword_of_weight(_sym), cpp/distfind/mitm.cpp:201-316 */
static int mitm_level(const mitm_view* v, int d) {
    const int nR = v->ncoord - v->nL;
    for (int wL = 0; wL <= d; ++wL) {
        const int wR = d - wL;
        if (wL > v->nL || wR > nR) continue;
        size_t nl, nr;
        u64* L = mitm_parts(v, 0, v->nL, wL, &nl);
        u64* R = mitm_parts(v, v->nL, nR, wR, &nr);
        mitm_kw = v->kw;
        qsort(L, nl, (size_t)v->kw * sizeof(u64), cmp_rec);
        int hit = 0;
        for (size_t i = 0; i < nr && !hit; ++i) {
            const u64* r = R + i * v->kw;
            /* first left record with syndrome >= r's */
            size_t lo = 0, hi = nl;
            while (lo < hi) {
                const size_t mid = (lo + hi) / 2;
                int c = 0;
                for (int q = 0; q < v->sw && !c; ++q) {
                    const u64 a = L[mid * v->kw + q], b = r[q];
                    c = a < b ? -1 : (a > b ? 1 : 0);
                }
                if (c < 0) lo = mid + 1; else hi = mid;
            }
            for (size_t j = lo; j < nl && !hit; ++j) {
                const u64* l = L + j * v->kw;
                int same = 1;
                for (int q = 0; q < v->sw && same; ++q) same = l[q] == r[q];
                if (!same) break;
                if (v->count_all) { hit = 1; break; }
                for (int q = v->sw; q < v->sw + v->lw; ++q)
                    if (l[q] != r[q]) { hit = 1; break; }
            }
        }
        free(L);
        free(R);
        if (hit) return 1;
    }
    return 0;
}

typedef struct {
    int has, target, seed_upper, found, level, resolved, confirmed;
    mitm_view v;
} mitm_side;

static void mitm_side_init(mitm_side* s, const problem* p) {
    memset(s, 0, sizeof(*s));
    s->found = -1;
    s->has = !(p->gen.rows == 0 || (!p->count_all && p->check.rows == 0));
    if (!s->has) { s->resolved = s->confirmed = 1; return; }
    s->v = mitm_view_of(p);
    s->seed_upper = p->seed_upper;
    s->target = p->seed_upper > 0 ? (p->seed_upper < s->v.ncoord ? p->seed_upper : s->v.ncoord)
                                  : s->v.ncoord;
}

static void mitm_side_free(mitm_side* s) {
    if (s->has) free(s->v.cols);
}

/* mitm_distance, cpp/distfind/mitm.cpp:318-380 */
static void mitm_single(const problem* p, orc_result* r) {
    memset(r, 0, sizeof(*r));
    mitm_side s;
    mitm_side_init(&s, p);
    if (s.has) {
        for (int d = 1; d <= s.target; ++d) {
            ++s.level;
            if (mitm_level(&s.v, d)) { s.found = d; break; }
        }
        if (s.found < 0 && s.seed_upper > 0 && s.target == s.seed_upper) s.found = s.seed_upper;
    }
    r->distance = s.found;
    r->levels = s.level;
    r->lower_bound = s.found >= 0 ? s.found : 0;
    r->proven = s.found >= 0;
    mitm_side_free(&s);
}

/* mitm_min_interleaved with cap_to_min, cpp/distfind/mitm.cpp:447-521 */
static void mitm_min(const problem* pz, const problem* px, orc_result* r) {
    memset(r, 0, sizeof(*r));
    mitm_side Z, X;
    mitm_side_init(&Z, pz);
    mitm_side_init(&X, px);
    mitm_side* sides[2] = {&Z, &X};
    int best = ORC_WEIGHT_NONE;
    if (Z.has && Z.seed_upper > 0 && Z.seed_upper < best) best = Z.seed_upper;
    if (X.has && X.seed_upper > 0 && X.seed_upper < best) best = X.seed_upper;
    const int tz = Z.has ? Z.target : 0, tx = X.has ? X.target : 0;
    const int maxd = tz > tx ? tz : tx;
    for (int d = 1; d <= maxd; ++d) {
        for (int k = 0; k < 2; ++k) {
            mitm_side* S = sides[k];
            if (S->resolved) continue;
            if (d > S->target) {
                if (S->seed_upper > 0 && S->target == S->seed_upper) {
                    S->found = S->seed_upper;
                    S->confirmed = 1;
                    if (S->found < best) best = S->found;
                }
                S->resolved = 1;
                continue;
            }
            if (d >= best) {
                S->confirmed = 1;
                if (S->seed_upper > 0 && best == S->seed_upper) S->found = best;
                S->resolved = 1;
                continue;
            }
            ++S->level;
            if (mitm_level(&S->v, d)) {
                S->found = d;
                if (d < best) best = d;
                S->confirmed = 1;
                S->resolved = 1;
            }
        }
        if (Z.resolved && X.resolved) break;
    }
    const int vz = Z.found >= 0 ? Z.found : ORC_WEIGHT_NONE;
    const int vx = X.found >= 0 ? X.found : ORC_WEIGHT_NONE;
    const int dist = vz < vx ? vz : vx;
    r->distance = dist >= ORC_WEIGHT_NONE ? -1 : dist;
    r->lower_bound = dist >= ORC_WEIGHT_NONE ? 0 : dist;
    r->levels = Z.level > X.level ? Z.level : X.level;
    r->proven = Z.confirmed && X.confirmed && dist < ORC_WEIGHT_NONE;
    mitm_side_free(&Z);
    mitm_side_free(&X);
}

/* the method switch of cpp/distfind/capi.cpp:53-60: "mitm" or BZ */
static void solve_single(const problem* p, const orc_options* opt, orc_result* r) {
    if (opt && opt->mitm) mitm_single(p, r); else bz_single(p, opt, r);
}
static void solve_min(const problem* pz, const problem* px, const orc_options* opt,
                      orc_result* r) {
    if (opt && opt->mitm) mitm_min(pz, px, r); else bz_min(pz, px, opt, r);
}

/* ------------------------------------------------------------------ public entry points */
int orc_classical_distance(const uint8_t* H, int rows, int cols, const orc_options* opt,
                           orc_result* out) {
    mat h = m_from_dense(H, rows, cols);
    problem p = classical_problem(&h);
    solve_single(&p, opt, out);
    p_free(&p);
    m_free(&h);
    return 0;
}

static int css_like(mat* A, mat* B, int subsystem, char which, const orc_options* opt,
                    orc_result* out) {
    if (which == 'Z' || which == 'X') {
        problem p = subsystem ? subsystem_problem(A, B, which)
                              : (which == 'X' ? build(B, A) : build(A, B));
        solve_single(&p, opt, out);
        p_free(&p);
    } else if (subsystem) {
        /* not interleaved, cpp/distfind/capi.cpp:256-274 */
        problem pz = subsystem_problem(A, B, 'Z'), px = subsystem_problem(A, B, 'X');
        orc_result rz, rx;
        solve_single(&pz, opt, &rz);
        solve_single(&px, opt, &rx);
        const int vz = rz.distance < 0 ? (1 << 30) : rz.distance;
        const int vx = rx.distance < 0 ? (1 << 30) : rx.distance;
        *out = vx < vz ? rx : rz;
        out->distance = vz < vx ? vz : vx;
        if (out->distance >= (1 << 30)) out->distance = -1;
        out->lower_bound = rz.lower_bound < rx.lower_bound ? rz.lower_bound : rx.lower_bound;
        out->proven = rz.proven && rx.proven;
        out->codewords = rz.codewords + rx.codewords;
        p_free(&pz);
        p_free(&px);
    } else {
        problem pz = build(A, B), px = build(B, A);
        solve_min(&pz, &px, opt, out);
        p_free(&pz);
        p_free(&px);
    }
    return 0;
}

int orc_css_distance(const uint8_t* Hx, int hxr, int hxc, const uint8_t* Hz, int hzr, int hzc,
                     char which, const orc_options* opt, orc_result* out) {
    mat A = m_from_dense(Hx, hxr, hxc), B = m_from_dense(Hz, hzr, hzc);
    css_like(&A, &B, 0, which, opt, out);
    m_free(&A);
    m_free(&B);
    return 0;
}

int orc_subsystem_distance(const uint8_t* Gx, int gxr, int gxc, const uint8_t* Gz, int gzr,
                           int gzc, char which, const orc_options* opt, orc_result* out) {
    mat A = m_from_dense(Gx, gxr, gxc), B = m_from_dense(Gz, gzr, gzc);
    css_like(&A, &B, 1, which, opt, out);
    m_free(&A);
    m_free(&B);
    return 0;
}

/* cpp/distfind/op_weight.cpp:9-36 */
static int coset_weight(const mat* G, const uint8_t* vec, const orc_options* opt) {
    u64* v = pack_vec(vec, G->cols);
    int res;
    if (in_rowspace_packed(G, v)) {
        res = 0;
    } else {
        problem p = coset_problem(G, v);
        orc_result r;
        solve_single(&p, opt, &r);
        res = r.distance;
        p_free(&p);
    }
    free(v);
    return res;
}

int orc_operator_weight(const uint8_t* Gx, int gxr, int gxc, const uint8_t* Gz, int gzr, int gzc,
                        const uint8_t* z, const uint8_t* x, const orc_options* opt, int* zw,
                        int* xw) {
    mat A = m_from_dense(Gx, gxr, gxc), B = m_from_dense(Gz, gzr, gzc);
    *zw = coset_weight(&B, z, opt);
    *xw = coset_weight(&A, x, opt);
    m_free(&A);
    m_free(&B);
    return 0;
}

/* symplectic_distance_driver, cpp/distfind/capi.cpp:168-223 (bz only) */
int orc_stabilizer_distance(const uint8_t* S, int rows, int cols, int subsystem, char which,
                            const orc_options* opt, orc_result* out) {
    if (cols % 2) return 2;
    mat G = m_from_dense(S, rows, cols);
    if (is_css(&G)) {
        mat Hx, Hz;
        split_css(&G, &Hx, &Hz);
        css_like(&Hx, &Hz, subsystem, which, opt, out);
        m_free(&Hx);
        m_free(&Hz);
        m_free(&G);
        return 0;
    }
    mat Sn = subsystem ? sympl_center(&G) : m_copy(&G);
    problem sp = sympl_problem(&Sn, &G);
    if (opt && opt->mitm) {
        /* mitm enumerates symplectic parts directly (cpp/distfind/capi.cpp:217-218) */
        mitm_single(&sp, out);
        p_free(&sp);
        m_free(&Sn);
        m_free(&G);
        return 0;
    }
    problem e = isometry(&sp);
    bz_single(&e, opt, out);
    if (out->distance > 0) out->distance /= 2;
    if (out->lower_bound > 0) out->lower_bound /= 2;
    p_free(&e);
    p_free(&sp);
    m_free(&Sn);
    m_free(&G);
    return 0;
}

int orc_pauli_operator_weight(const uint8_t* Gm, int rows, int cols, const uint8_t* op,
                              const orc_options* opt, orc_result* out) {
    if (cols % 2) return 2;
    memset(out, 0, sizeof(*out));
    mat G = m_from_dense(Gm, rows, cols);
    u64* v = pack_vec(op, cols);
    if (in_rowspace_packed(&G, v)) {
        out->distance = 0;
        out->proven = 1;
    } else {
        problem p = coset_problem(&G, v);
        p.symplectic = 1;
        p.qubits = cols / 2;
        p.seed_upper = sw_weight(v, p.qubits);
        if (opt && opt->mitm) {
            mitm_single(&p, out);   /* cpp/distfind/capi.cpp:272-282 */
        } else {
            problem e = isometry(&p);
            bz_single(&e, opt, out);
            if (out->distance > 0) out->distance /= 2;
            if (out->lower_bound > 0) out->lower_bound /= 2;
            p_free(&e);
        }
        p_free(&p);
    }
    free(v);
    m_free(&G);
    return 0;
}

int orc_prepare(int kind, const uint8_t* A, int ar, int ac, const uint8_t* B, int br, int bc,
                int* meta, int* ranks, int max_gamma) {
    mat a = m_from_dense(A, ar, ac);
    mat b = (B && br > 0) ? m_from_dense(B, br, bc) : m_new(0, ac);
    problem p;
    switch (kind) {
        case 0: p = classical_problem(&a); break;
        case 1: p = build(&a, &b); break;
        case 2: p = build(&b, &a); break;
        case 3: p = subsystem_problem(&a, &b, 'Z'); break;
        case 4: p = subsystem_problem(&a, &b, 'X'); break;
        default: {
            problem sp = sympl_problem(&a, &a);
            p = isometry(&sp);
            p_free(&sp);
        }
    }
    gseq q = {0};
    if (p.gen.rows > 0) { q = gamma_sequence(&p.gen); sort_by_rank(&q); }
    meta[0] = p.n; meta[1] = p.gen.rows; meta[2] = q.n;
    meta[3] = p.count_all ? 0 : p.check.rows;
    meta[4] = p.even; meta[5] = p.count_all; meta[6] = p.seed_upper;
    meta[7] = words_for(p.n);
    for (int g = 0; g < q.n && g < max_gamma; ++g) ranks[g] = q.s[g].rank;
    gs_free(&q);
    p_free(&p);
    m_free(&a);
    m_free(&b);
    return 0;
}

/* ------------------------------------------------------------------ codeaut collection
 * The low-weight collector behind codeaut_bz_collect (cpp/codeaut/bz.cpp:55-117): for every
 * subset size sw = 1..min(p, m) every sw-subset of G's rows is XORed, and the results of
 * weight 1..keep are kept (the CollectSink of cpp/qsf/enum_core.hpp:90-103: weight 0, a
 * dependent subset, is never kept); the kept rows are then sorted by their packed words,
 * word 0 first (RowLess, bz.cpp:38-50), and duplicates dropped.  The combination count
 * saturates at 2^62 per level and in total (COMBO_CAP, bz.cpp:29, 87-97).  Subsets are
 * visited in the reference's lexicographic order (next_comb, cpp/qsf/combinatorics.hpp:
 * 64-71); acc[i] holds the XOR of the rows pos[0..i]. */
static int orc_stride_words;
static int cmp_rows(const void* a, const void* b) {
    const u64* x = (const u64*)a;
    const u64* y = (const u64*)b;
    for (int i = 0; i < orc_stride_words; ++i)
        if (x[i] != y[i]) return x[i] < y[i] ? -1 : 1;
    return 0;
}

long long orc_collect(const uint8_t* G, int m, int n, int p, int keep, uint64_t** out,
                      long long* combos) {
    const long long cap62 = (long long)1 << 62;
    *out = NULL;
    *combos = 0;
    if (m <= 0 || n <= 0 || p <= 0) return 0;
    const int s = words_for(n);
    mat rows = m_from_dense(G, m, n);
    const int maxsw = p < m ? p : m;
    size_t nh = 0, caph = 1024;
    u64* hits = (u64*)malloc(caph * s * sizeof(u64));
    u64* acc = (u64*)calloc((size_t)maxsw * s, sizeof(u64));
    int* pos = (int*)malloc(sizeof(int) * (size_t)maxsw);
    if (!hits || !acc || !pos) { free(hits); free(acc); free(pos); m_free(&rows); return -1; }
    for (int sw = 1; sw <= maxsw; ++sw) {
        /* C(m, sw) with the reference's saturation */
        unsigned long long c = 1;
        int sat = 0;
        for (int i = 1; i <= sw && !sat; ++i) {
            unsigned __int128 t = (unsigned __int128)c * (unsigned)(m - sw + i) / (unsigned)i;
            if (t > (unsigned __int128)cap62) sat = 1; else c = (unsigned long long)t;
        }
        const long long total = sat ? cap62 : (long long)c;
        *combos = (*combos > cap62 - total) ? cap62 : *combos + total;
        for (int i = 0; i < sw; ++i) pos[i] = i;
        int from = 0;   /* first position whose prefix XOR must be rebuilt */
        for (;;) {
            for (int i = from; i < sw; ++i) {
                u64* a = acc + (size_t)i * s;
                const u64* r = m_row(&rows, pos[i]);
                for (int w = 0; w < s; ++w) a[w] = (i ? acc[(size_t)(i - 1) * s + w] : 0) ^ r[w];
            }
            const u64* cw = acc + (size_t)(sw - 1) * s;
            const int wt = v_weight(cw, s);
            if (wt > 0 && wt <= keep) {
                if (nh == caph) {
                    caph *= 2;
                    u64* nhits = (u64*)realloc(hits, caph * s * sizeof(u64));
                    if (!nhits) { free(hits); free(acc); free(pos); m_free(&rows); return -1; }
                    hits = nhits;
                }
                memcpy(hits + nh * s, cw, (size_t)s * sizeof(u64));
                ++nh;
            }
            int j = sw - 1;
            while (j >= 0 && pos[j] == m - sw + j) --j;
            if (j < 0) break;
            ++pos[j];
            for (int t = j + 1; t < sw; ++t) pos[t] = pos[t - 1] + 1;
            from = j;
        }
    }
    orc_stride_words = s;
    if (nh > 1) qsort(hits, nh, (size_t)s * sizeof(u64), cmp_rows);
    size_t nu = 0;
    for (size_t i = 0; i < nh; ++i) {
        if (nu > 0 && memcmp(hits + (nu - 1) * s, hits + i * s, (size_t)s * sizeof(u64)) == 0)
            continue;
        if (nu != i) memcpy(hits + nu * s, hits + i * s, (size_t)s * sizeof(u64));
        ++nu;
    }
    free(acc);
    free(pos);
    m_free(&rows);
    *out = hits;
    return (long long)nu;
}

void orc_free(void* ptr) { free(ptr); }
