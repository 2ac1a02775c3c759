/*
 * Multi-row stack interpreter for fit records, forward and reverse: each
 * thread carries NR rows (f32 or f64) through one decode of every
 * instruction.
 *
 * A fit-record program (post-order records [op, kid0, kid1, slot],
 * my-version/src/fit.rs:985-1056) of a tree is evaluated on a stack exactly
 * like postfix bytecode. The host translates it once per batch into 8-byte
 * instructions: pushes of an input column or a constant slot, unary and
 * binary operators, and a binary operator fused with the push of its right
 * operand. The top of stack lives in registers (NR rows per thread),
 * deeper entries in shared-memory spill slots fixed at decode time.
 *
 * The reverse sweep is the mirror of the forward stack machine: an
 * operator's adjoint arrives on top of stack, its children's adjoints leave
 * through the same spill slot and top of stack their values used, so no
 * per-node value tape is needed. It runs over a second instruction list in
 * which every subtree without a constant is collapsed to the restore of the
 * adjoint below it (or dropped), since nothing in it has a constant to
 * differentiate. Only the local partials that lie on a path from a constant
 * to the root are kept, in a per-thread shared-memory tape. A zero adjoint
 * passes nothing to its operands, as the reference's adjoint does
 * (eval.cu:1245-1246, fit.rs:1479-1481).
 */
#pragma once

#include <cstring>
#include <vector>

#include "rc_ops.cuh"

enum FiKind {
    FI_PUSH_VAR = 0,   /* spill TOS to `spill`; TOS = x[imm]. Reverse: restore only */
    FI_PUSH_PARAM = 1, /* spill TOS; TOS = c[imm] */
    FI_PUSH_CACHE = 2, /* spill TOS; TOS = cached column imm of the candidate */
    FI_UNARY = 3,      /* TOS = op(TOS) */
    FI_BIN_S = 4,      /* TOS = op(slot[arg], TOS) */
    FI_BIN_V = 5,      /* TOS = op(TOS, x[imm]) */
    FI_BIN_P = 6,      /* TOS = op(TOS, c[imm]) */
    FI_HALT = 7
};

/* Flag bits above the kind: the left (or only) / right operand's subtree
   holds a constant, and a reverse store that adds to an earlier one. */
#define FI_KIND_MASK 7u
#define FI_HP_L 8u
#define FI_HP_R 16u
#define FI_ACC 32u

struct FIns {
    uint8_t kind;  /* FiKind | flags */
    uint8_t op;
    uint8_t arg;   /* spill slot of the left operand (FI_BIN_S) */
    uint8_t spill; /* slot a push spills TOS to, 0xff when the stack was empty */
    uint16_t imm;  /* input column or constant slot */
    uint16_t tape; /* first partial-tape slot of this instruction */
};
static_assert(sizeof(FIns) == 8, "FIns is 8 bytes");

__host__ __device__ constexpr bool fi_nonlinear(unsigned op)
{
    return op != OP_ADD && op != OP_SUB && op != OP_NEG;
}

/* Host translation of one fit-record program into the forward list `fwd`
   (ending in HALT) and the reverse list `rev` (walked last to first).
   Returns false when the records are not a tree in stack (post-) order,
   which the device path rejects.

   With `fwdc`, also the forward list in which every maximal constant-free
   subtree of two or more instructions is replaced by one push of a cached
   column (its values over all rows do not depend on the constants, so they
   are computed once per fit), and in `subs` the records of each such
   subtree, renumbered as a program of its own, in cache-column order.

   With `inputs`, the lists differentiate with respect to the inputs instead
   of the constants: the partials kept and the subtrees pruned are those on
   and off paths from an input leaf, a pruned left operand is restored by a
   push of kind FI_PUSH_CACHE, and the reverse sweep's input leaves (pushes
   and fused operands of kind FI_PUSH_VAR / FI_BIN_V) add their adjoints to
   the input's gradient (fi_reverse_x). No cached list is made. */
inline bool fi_decode(const uint32_t *rec, int m, std::vector<FIns> &fwd, std::vector<FIns> &rev,
                      int *nslots, int *ntape, std::vector<FIns> *fwdc = nullptr,
                      std::vector<std::vector<uint32_t>> *subs = nullptr, bool inputs = false)
{
    const uint32_t leaf_op = inputs ? OP_VAR : OP_CONST;
    struct Ent {
        int rec, first;
        bool hp;
    };
    std::vector<Ent> stack;
    std::vector<int> lo(m, 0), hi(m, -1), kid0(m, -1), kid1(m, -1), first_rec(m, 0);
    std::vector<char> hp(m, 0), fused(m, 0);
    int depth = 0, maxslot = -1, tape = 0;
    fwd.clear();
    rev.clear();
    for (int i = 0; i < m; ++i) {
        const uint32_t op = rec[4 * i], k0 = rec[4 * i + 1], k1 = rec[4 * i + 2],
                       slot = rec[4 * i + 3];
        FIns in;
        in.kind = 0;
        in.op = (uint8_t)op;
        in.arg = 0;
        in.spill = 0xff;
        in.imm = 0;
        in.tape = (uint16_t)tape;
        if (op == OP_CONST || op == OP_VAR) {
            if (slot > 0xffff || depth >= 250) return false;
            in.kind = op == OP_CONST ? FI_PUSH_PARAM : FI_PUSH_VAR;
            in.imm = (uint16_t)slot;
            if (depth >= 1) {
                in.spill = (uint8_t)(depth - 1);
                maxslot = maxslot > depth - 1 ? maxslot : depth - 1;
            }
            ++depth;
            hp[i] = op == leaf_op;
            first_rec[i] = i;
            lo[i] = (int)fwd.size();
            stack.push_back({i, (int)fwd.size(), op == leaf_op});
            fwd.push_back(in);
            hi[i] = lo[i];
        } else if (ft_op_binary(op)) {
            if (stack.size() < 2 || stack[stack.size() - 1].rec != (int)k1 ||
                stack[stack.size() - 2].rec != (int)k0)
                return false;
            const Ent L = stack[stack.size() - 2], R = stack[stack.size() - 1];
            stack.pop_back();
            const bool h = L.hp || R.hp;
            hp[i] = h;
            kid0[i] = (int)k0;
            kid1[i] = (int)k1;
            first_rec[i] = first_rec[k0];
            unsigned flags = 0;
            int np = 0;
            if (h) {
                flags = (L.hp ? FI_HP_L : 0u) | (R.hp ? FI_HP_R : 0u);
                if (fi_nonlinear(op)) np = (L.hp ? 1 : 0) + (R.hp ? 1 : 0);
            }
            in.kind = (uint8_t)(FI_BIN_S | flags);
            in.arg = (uint8_t)(depth - 2);
            --depth;
            FIns &prev = fwd.back();
            const unsigned pk = prev.kind & FI_KIND_MASK;
            if ((pk == FI_PUSH_VAR || pk == FI_PUSH_PARAM) && prev.spill == in.arg) {
                /* fuse "push right operand; op" */
                prev.kind = (uint8_t)((pk == FI_PUSH_VAR ? FI_BIN_V : FI_BIN_P) | flags);
                prev.op = (uint8_t)op;
                prev.spill = 0xff;
                prev.tape = (uint16_t)tape;
                fused[k1] = 1;
            } else {
                fwd.push_back(in);
            }
            tape += np;
            lo[i] = L.first;
            hi[i] = (int)fwd.size() - 1;
            stack.back() = {i, L.first, h};
        } else {
            if (stack.empty() || stack.back().rec != (int)k0) return false;
            const Ent C = stack.back();
            hp[i] = C.hp;
            kid0[i] = (int)k0;
            first_rec[i] = first_rec[k0];
            in.kind = (uint8_t)(FI_UNARY | (C.hp ? FI_HP_L : 0u));
            if (C.hp && fi_nonlinear(op)) ++tape;
            lo[i] = C.first;
            fwd.push_back(in);
            hi[i] = (int)fwd.size() - 1;
            stack.back() = {i, C.first, C.hp};
        }
        if (tape > 0xfff0) return false;
    }
    if (stack.size() != 1 || stack[0].rec != m - 1) return false;
    FIns h;
    h.kind = FI_HALT;
    h.op = 0;
    h.arg = 0;
    h.spill = 0xff;
    h.imm = 0;
    h.tape = (uint16_t)tape;
    fwd.push_back(h);
    *nslots = maxslot + 1;
    *ntape = tape;

    /* reverse list: maximal constant-free subtrees below a node with a
       constant become a restore of the adjoint below them (the left operand
       of a binary), or vanish (the right operand: its operator hands the left
       adjoint on directly; a fused leaf has no instruction of its own) */
    const int nf = (int)fwd.size() - 1;
    std::vector<int> skip_to(nf, -1);
    std::vector<char> emit(nf, 0);
    for (int i = 0; i < m; ++i) {
        if (!hp[i]) continue;
        const int kids[2] = {kid0[i], kid1[i]};
        for (int s = 0; s < 2; ++s) {
            const int k = kids[s];
            if (k < 0 || hp[k] || fused[k] || hi[k] < lo[k]) continue;
            skip_to[lo[k]] = hi[k];
            emit[lo[k]] = (s == 0 && fwd[lo[k]].spill != 0xff) ? 1 : 0;
        }
    }
    if (hp[m - 1]) {
        for (int j = 0; j < nf;) {
            if (skip_to[j] >= 0) {
                if (emit[j]) {
                    FIns r = fwd[j];
                    r.kind = inputs ? FI_PUSH_CACHE : FI_PUSH_VAR;
                    rev.push_back(r);
                }
                j = skip_to[j] + 1;
            } else {
                rev.push_back(fwd[j]);
                ++j;
            }
        }
    }
    /* a constant slot met again (in reverse order) accumulates */
    std::vector<char> seen(65536, 0);
    for (int j = (int)rev.size() - 1; j >= 0; --j) {
        const unsigned k = rev[j].kind & FI_KIND_MASK;
        if (k == FI_PUSH_PARAM || k == FI_BIN_P) {
            if (seen[rev[j].imm]) rev[j].kind |= FI_ACC;
            seen[rev[j].imm] = 1;
        }
    }
    if (inputs) return true;
    if (fwdc) {
        /* cacheable: constant-free, its own instructions (not a fused leaf),
           two or more of them, and its parent has a constant (or it is the
           whole tree) */
        std::vector<int> parent(m, -1);
        for (int i = 0; i < m; ++i) {
            if (kid0[i] >= 0) parent[kid0[i]] = i;
            if (kid1[i] >= 0) parent[kid1[i]] = i;
        }
        std::vector<int> start_of(nf, -1);
        for (int k = 0; k < m; ++k) {
            if (hp[k] || fused[k] || hi[k] - lo[k] < 1) continue;
            if (parent[k] >= 0 && !hp[parent[k]]) continue;
            start_of[lo[k]] = k;
        }
        fwdc->clear();
        if (subs) subs->clear();
        int col = 0;
        for (int j = 0; j < nf;) {
            const int k = start_of[j];
            if (k < 0) {
                fwdc->push_back(fwd[j]);
                ++j;
                continue;
            }
            FIns c = fwd[j];
            c.kind = FI_PUSH_CACHE;
            c.op = 0;
            c.arg = 0;
            c.imm = (uint16_t)col++;
            c.tape = 0;
            fwdc->push_back(c);
            if (subs) {
                const int b = first_rec[k];
                std::vector<uint32_t> s(4 * (size_t)(k - b + 1));
                for (int r = b; r <= k; ++r) {
                    const uint32_t op = rec[4 * r];
                    const bool leaf = op == OP_CONST || op == OP_VAR;
                    const bool bin = !leaf && ft_op_binary(op);
                    s[4 * (r - b) + 0] = op;
                    s[4 * (r - b) + 1] = leaf ? rec[4 * r + 1] : rec[4 * r + 1] - (uint32_t)b;
                    s[4 * (r - b) + 2] = bin ? rec[4 * r + 2] - (uint32_t)b : rec[4 * r + 2];
                    s[4 * (r - b) + 3] = rec[4 * r + 3];
                }
                subs->push_back(std::move(s));
            }
            j = hi[k] + 1;
        }
        fwdc->push_back(fwd[nf]);
    }
    return true;
}

/* Local partials of one operator (ft_partials_f / ft_partials_d semantics,
   with the operator's value `r` reused where it is the same expression). A
   `pow` with a non-positive base passes nothing. */
template <typename V>
__device__ __forceinline__ void fi_partials(unsigned op, V x, V y, V r, V &d0, V &d1)
{
    d0 = V(0);
    d1 = V(0);
    switch (op) {
        case OP_EXP: d0 = r; break;
        case OP_LOG: d0 = V(1) / x; break;
        case OP_ABS: d0 = x >= V(0) ? V(1) : V(-1); break;
        case OP_SQRT: d0 = V(1) / (V(2) * r); break;
        case OP_SIN: d0 = cos(x); break;
        case OP_COS: d0 = -sin(x); break;
        case OP_TAN: {
            const V t = cos(x);
            d0 = V(1) / (t * t);
        } break;
        case OP_SINH: d0 = cosh(x); break;
        case OP_COSH: d0 = sinh(x); break;
        case OP_TANH: d0 = V(1) - r * r; break;
        case OP_SIG: d0 = r * (V(1) - r); break;
        case OP_GAUSS: d0 = (V(-2) * x) * r; break;
        case OP_SQUARE: d0 = V(2) * x; break;
        case OP_CUBE: d0 = V(3) * x * x; break;
        case OP_ERF: d0 = V(1.1283791670955126) * exp(-x * x); break;
        case OP_ERFC: d0 = V(-1.1283791670955126) * exp(-x * x); break;
        case OP_MUL: d0 = y; d1 = x; break;
        case OP_DIV: d0 = V(1) / y; d1 = -x / (y * y); break;
        case OP_POW:
            if (x > V(0)) {
                d0 = y * pow(x, y - V(1));
                d1 = r * log(x);
            }
            break;
        default: break;
    }
}

/* The rows a thread carries: NR values of type V, moved as one 4-, 8- or
   16-byte vector (spill slots, tape, column loads). */
template <typename V, int NR>
struct FiV {
    struct alignas(sizeof(V) * NR) V4 {
        V v[NR];
    };
    __device__ __forceinline__ static void unpack(const V4 &x, V *v)
    {
#pragma unroll
        for (int i = 0; i < NR; ++i) v[i] = x.v[i];
    }
    __device__ __forceinline__ static V4 pack(const V *v)
    {
        V4 x;
#pragma unroll
        for (int i = 0; i < NR; ++i) x.v[i] = v[i];
        return x;
    }
    /* read-only load of NR consecutive column values */
    __device__ __forceinline__ static void ldg(const V *p, V *v)
    {
        V4 x;
        if constexpr (sizeof(V4) == 16) {
            const float4 t = __ldg(reinterpret_cast<const float4 *>(p));
            memcpy(&x, &t, 16);
        } else if constexpr (sizeof(V4) == 8) {
            const float2 t = __ldg(reinterpret_cast<const float2 *>(p));
            memcpy(&x, &t, 8);
        } else {
            const float t = __ldg(reinterpret_cast<const float *>(p));
            memcpy(&x, &t, 4);
        }
        unpack(x, v);
    }
    __device__ __forceinline__ static V value(unsigned op, V a, V b)
    {
        if constexpr (sizeof(V) == 8) return ft_value_d(op, a, b);
        else return ft_value_f(op, a, b);
    }
};

template <typename V>
__device__ __forceinline__ V fi_child(V a, V d)
{
    return a == V(0) ? V(0) : a * d;
}

/* One operator on the thread's rows: values, and with PARTIALS the
   partials the instruction keeps. The operator is a compile-time constant in
   each case, so the value and partial switches fold away. */
#define FI_OPN(OPC)                                                                   \
    case OPC: {                                                                       \
        _Pragma("unroll") for (int i = 0; i < NR; ++i) r[i] = F::value(OPC, a[i], b[i]); \
        if (PARTIALS && fi_nonlinear(OPC) && (kind & (FI_HP_L | FI_HP_R))) {          \
            V pl[NR], pr[NR];                                                         \
            _Pragma("unroll") for (int i = 0; i < NR; ++i)                            \
                fi_partials<V>(OPC, a[i], b[i], r[i], pl[i], pr[i]);                  \
            int ts = in.tape;                                                         \
            if (kind & FI_HP_L) {                                                     \
                tape[ts * S + tid] = F::pack(pl);                             \
                ++ts;                                                                 \
            }                                                                         \
            if (kind & FI_HP_R) tape[ts * S + tid] = F::pack(pr);             \
        }                                                                             \
    } break;

/* Forward sweep of the thread's NR rows. Constants from `cf`, inputs from
   the columns at `row` (aligned to the row vector), cached subtree values
   from `ccols` (same stride). Spill slots and the tape are [slot][S] row
   vectors with this thread at `tid`. The prediction of row i is left in
   out[i]. */
template <typename V, int NR, bool PARTIALS>
__device__ __forceinline__ void fi_forward(const FIns *__restrict__ prog, const V *cf,
                                           const V *__restrict__ cols, int npad, int row,
                                           typename FiV<V, NR>::V4 *stk,
                                           typename FiV<V, NR>::V4 *tape, int S, int tid, V *out,
                                           const V *__restrict__ ccols = nullptr)
{
    using F = FiV<V, NR>;
    V t[NR];
#pragma unroll
    for (int i = 0; i < NR; ++i) t[i] = V(0);
    for (int pc = 0; pc < 512; ++pc) {
        const FIns in = prog[pc];
        const unsigned kind = in.kind;
        const unsigned k = kind & FI_KIND_MASK;
        if (k <= FI_PUSH_CACHE) {
            if (in.spill != 0xff) stk[in.spill * S + tid] = F::pack(t);
            if (k == FI_PUSH_VAR) {
                F::ldg(cols + (size_t)in.imm * (size_t)npad + row, t);
            } else if (k == FI_PUSH_CACHE) {
                F::ldg(ccols + (size_t)in.imm * (size_t)npad + row, t);
            } else {
                const V c = cf[in.imm];
#pragma unroll
                for (int i = 0; i < NR; ++i) t[i] = c;
            }
            continue;
        }
        if (k == FI_HALT) break;
        V a[NR], b[NR];
        if (k == FI_BIN_S) {
            F::unpack(stk[in.arg * S + tid], a);
#pragma unroll
            for (int i = 0; i < NR; ++i) b[i] = t[i];
        } else {
#pragma unroll
            for (int i = 0; i < NR; ++i) {
                a[i] = t[i];
                b[i] = V(0);
            }
            if (k == FI_BIN_V) {
                F::ldg(cols + (size_t)in.imm * (size_t)npad + row, b);
            } else if (k == FI_BIN_P) {
                const V c = cf[in.imm];
#pragma unroll
                for (int i = 0; i < NR; ++i) b[i] = c;
            }
        }
        V r[NR];
        switch (in.op) {
            FI_OPN(OP_ADD) FI_OPN(OP_SUB) FI_OPN(OP_MUL) FI_OPN(OP_DIV) FI_OPN(OP_POW)
            case OP_SIN:
            case OP_COS:
                if (sizeof(V) == 4 && PARTIALS && (kind & FI_HP_L)) {
                    /* one f32 sincosf gives the value and the partial (its
                       results equal sinf / cosf bit for bit on B200) */
                    V pl[NR];
                    const bool is_sin = in.op == OP_SIN;
#pragma unroll
                    for (int i = 0; i < NR; ++i) {
                        float s, c;
                        sincosf((float)a[i], &s, &c);
                        r[i] = is_sin ? s : c;
                        pl[i] = is_sin ? c : -s;
                    }
                    tape[in.tape * S + tid] = F::pack(pl);
                } else if (in.op == OP_SIN) {
#pragma unroll
                    for (int i = 0; i < NR; ++i) r[i] = F::value(OP_SIN, a[i], b[i]);
                    if (PARTIALS && (kind & FI_HP_L)) {
                        V pl[NR];
#pragma unroll
                        for (int i = 0; i < NR; ++i) pl[i] = cos(a[i]);
                        tape[in.tape * S + tid] = F::pack(pl);
                    }
                } else {
#pragma unroll
                    for (int i = 0; i < NR; ++i) r[i] = F::value(OP_COS, a[i], b[i]);
                    if (PARTIALS && (kind & FI_HP_L)) {
                        V pl[NR];
#pragma unroll
                        for (int i = 0; i < NR; ++i) pl[i] = -sin(a[i]);
                        tape[in.tape * S + tid] = F::pack(pl);
                    }
                }
                break;
            FI_OPN(OP_TAN) FI_OPN(OP_EXP) FI_OPN(OP_LOG)
            FI_OPN(OP_SQRT) FI_OPN(OP_ABS) FI_OPN(OP_TANH) FI_OPN(OP_SIG) FI_OPN(OP_SQUARE)
            FI_OPN(OP_CUBE) FI_OPN(OP_NEG) FI_OPN(OP_GAUSS) FI_OPN(OP_SINH) FI_OPN(OP_COSH)
            FI_OPN(OP_ERF) FI_OPN(OP_ERFC)
            default:
#pragma unroll
                for (int i = 0; i < NR; ++i) r[i] = V(NAN);
                break;
        }
#pragma unroll
        for (int i = 0; i < NR; ++i) t[i] = r[i];
    }
#pragma unroll
    for (int i = 0; i < NR; ++i) out[i] = t[i];
}
#undef FI_OPN

/* Reverse sweep of the thread's rows over the reverse list (`nr` entries,
   walked from the last). The adjoints start at the rows' seeds `a`.
   Constant adjoints are stored to g[slot * R + i * A] for row i (`g` is
   this thread's first row). Returns whether every stored value is
   finite. */
template <typename V, int NR>
__device__ __forceinline__ bool fi_reverse(const FIns *__restrict__ rev, int nr,
                                           typename FiV<V, NR>::V4 *stk,
                                           const typename FiV<V, NR>::V4 *tape, int S, int tid,
                                           V *g, int R, int A, V *a)
{
    using F = FiV<V, NR>;
    bool fin = true;
    for (int pc = nr - 1; pc >= 0; --pc) {
        const FIns in = rev[pc];
        const unsigned kind = in.kind;
        const unsigned k = kind & FI_KIND_MASK;
        if (k <= FI_PUSH_CACHE) {
            if (k == FI_PUSH_PARAM) {
                V *gs = g + in.imm * R;
#pragma unroll
                for (int i = 0; i < NR; ++i) {
                    const V v = (kind & FI_ACC) ? a[i] + gs[i * A] : a[i];
                    gs[i * A] = v;
                    fin = fin && isfinite(v);
                }
            }
            if (in.spill != 0xff) F::unpack(stk[in.spill * S + tid], a);
            continue;
        }
        if (k == FI_UNARY) {
            if (in.op == OP_NEG) {
#pragma unroll
                for (int i = 0; i < NR; ++i) a[i] = -a[i];
            } else {
                V d[NR];
                F::unpack(tape[in.tape * S + tid], d);
#pragma unroll
                for (int i = 0; i < NR; ++i) a[i] = fi_child(a[i], d[i]);
            }
            continue;
        }
        /* binary: left adjoint l, right adjoint r, for the sides with a
           constant */
        V l[NR], r[NR];
        if (in.op == OP_ADD || in.op == OP_SUB) {
            const bool sub = in.op == OP_SUB;
#pragma unroll
            for (int i = 0; i < NR; ++i) {
                l[i] = a[i];
                r[i] = sub ? -a[i] : a[i];
            }
        } else {
            int ts = in.tape;
#pragma unroll
            for (int i = 0; i < NR; ++i) l[i] = r[i] = V(0);
            if (kind & FI_HP_L) {
                V d[NR];
                F::unpack(tape[ts * S + tid], d);
#pragma unroll
                for (int i = 0; i < NR; ++i) l[i] = fi_child(a[i], d[i]);
                ++ts;
            }
            if (kind & FI_HP_R) {
                V d[NR];
                F::unpack(tape[ts * S + tid], d);
#pragma unroll
                for (int i = 0; i < NR; ++i) r[i] = fi_child(a[i], d[i]);
            }
        }
        if (k == FI_BIN_S) {
            if ((kind & FI_HP_L) && (kind & FI_HP_R)) {
                /* the left adjoint waits in its spill slot while the right
                   subtree is walked; that subtree's first push restores it */
                stk[in.arg * S + tid] = F::pack(l);
#pragma unroll
                for (int i = 0; i < NR; ++i) a[i] = r[i];
            } else if (kind & FI_HP_R) {
#pragma unroll
                for (int i = 0; i < NR; ++i) a[i] = r[i];
            } else {
#pragma unroll
                for (int i = 0; i < NR; ++i) a[i] = l[i];
            }
        } else {
            if (k == FI_BIN_P) {
                V *gs = g + in.imm * R;
#pragma unroll
                for (int i = 0; i < NR; ++i) {
                    const V v = (kind & FI_ACC) ? r[i] + gs[i * A] : r[i];
                    gs[i * A] = v;
                    fin = fin && isfinite(v);
                }
            }
#pragma unroll
            for (int i = 0; i < NR; ++i) a[i] = l[i];
        }
    }
    return fin;
}

/* Reverse sweep of the thread's rows over an input-mode reverse list (see
   fi_decode): the same stack machine as fi_reverse, seeded with a[], whose
   input leaves add their adjoints to the thread's gradient rows
   ig[col * S + tid] (zeroed by the caller). Constants receive nothing. */
template <typename V, int NR>
__device__ __forceinline__ void fi_reverse_x(const FIns *__restrict__ rev, int nr,
                                             typename FiV<V, NR>::V4 *stk,
                                             const typename FiV<V, NR>::V4 *tape, int S, int tid,
                                             typename FiV<V, NR>::V4 *ig, V *a)
{
    using F = FiV<V, NR>;
    for (int pc = nr - 1; pc >= 0; --pc) {
        const FIns in = rev[pc];
        const unsigned kind = in.kind;
        const unsigned k = kind & FI_KIND_MASK;
        if (k <= FI_PUSH_CACHE) {
            if (k == FI_PUSH_VAR) {
                V gv[NR];
                F::unpack(ig[in.imm * S + tid], gv);
#pragma unroll
                for (int i = 0; i < NR; ++i) gv[i] += a[i];
                ig[in.imm * S + tid] = F::pack(gv);
            }
            if (in.spill != 0xff) F::unpack(stk[in.spill * S + tid], a);
            continue;
        }
        if (k == FI_UNARY) {
            if (in.op == OP_NEG) {
#pragma unroll
                for (int i = 0; i < NR; ++i) a[i] = -a[i];
            } else {
                V d[NR];
                F::unpack(tape[in.tape * S + tid], d);
#pragma unroll
                for (int i = 0; i < NR; ++i) a[i] = fi_child(a[i], d[i]);
            }
            continue;
        }
        V l[NR], r[NR];
        if (in.op == OP_ADD || in.op == OP_SUB) {
            const bool sub = in.op == OP_SUB;
#pragma unroll
            for (int i = 0; i < NR; ++i) {
                l[i] = a[i];
                r[i] = sub ? -a[i] : a[i];
            }
        } else {
            int ts = in.tape;
#pragma unroll
            for (int i = 0; i < NR; ++i) l[i] = r[i] = V(0);
            if (kind & FI_HP_L) {
                V d[NR];
                F::unpack(tape[ts * S + tid], d);
#pragma unroll
                for (int i = 0; i < NR; ++i) l[i] = fi_child(a[i], d[i]);
                ++ts;
            }
            if (kind & FI_HP_R) {
                V d[NR];
                F::unpack(tape[ts * S + tid], d);
#pragma unroll
                for (int i = 0; i < NR; ++i) r[i] = fi_child(a[i], d[i]);
            }
        }
        if (k == FI_BIN_S) {
            if ((kind & FI_HP_L) && (kind & FI_HP_R)) {
                stk[in.arg * S + tid] = F::pack(l);
#pragma unroll
                for (int i = 0; i < NR; ++i) a[i] = r[i];
            } else if (kind & FI_HP_R) {
#pragma unroll
                for (int i = 0; i < NR; ++i) a[i] = r[i];
            } else {
#pragma unroll
                for (int i = 0; i < NR; ++i) a[i] = l[i];
            }
        } else {
            if (k == FI_BIN_V) {
                V gv[NR];
                F::unpack(ig[in.imm * S + tid], gv);
#pragma unroll
                for (int i = 0; i < NR; ++i) gv[i] += r[i];
                ig[in.imm * S + tid] = F::pack(gv);
            }
#pragma unroll
            for (int i = 0; i < NR; ++i) a[i] = l[i];
        }
    }
}

/* D = A * B + D for one 8x8x4 f64 tile (mma.sync; A row-major, B
   column-major). Lane (g = lane / 4, t = lane % 4) holds A[g][t], B[t][g]
   and D[g][2t], D[g][2t + 1]. */
__device__ __forceinline__ void fi_dmma(double &d0, double &d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}
