/*
 * Four-rows-per-thread stack interpreter for fit records, forward and
 * reverse.
 *
 * A fit-record program (post-order records [op, kid0, kid1, slot],
 * my-version/src/fit.rs:985-1056) of a tree is evaluated on a stack exactly
 * like postfix bytecode. The host translates it once per batch into 8-byte
 * instructions: pushes of an input column or a constant slot, unary and
 * binary operators, and a binary operator fused with the push of its right
 * operand. The top of stack lives in registers (four rows per thread,
 * `float4`), deeper entries in shared-memory spill slots fixed at decode time.
 *
 * The reverse sweep walks the instructions backwards and is the mirror of the
 * forward stack machine: an operator's adjoint arrives on top of stack, its
 * children's adjoints leave through the same spill slot and top of stack
 * their values used, so no per-node value tape is needed. Only the local
 * partial derivatives of non-linear operators are kept, in a per-thread
 * shared-memory tape (one slot per partial). A zero adjoint passes nothing
 * to its operands, as the reference's adjoint does (eval.cu:1245-1246,
 * fit.rs:1479-1481).
 */
#pragma once

#include <vector>

#include "rc_ops.cuh"

enum FiKind {
    FI_PUSH_VAR = 0,   /* spill TOS to `spill`; TOS = x[imm] */
    FI_PUSH_PARAM = 1, /* spill TOS; TOS = c[imm] */
    FI_UNARY = 2,      /* TOS = op(TOS) */
    FI_BIN_S = 3,      /* TOS = op(slot[arg], TOS) */
    FI_BIN_V = 4,      /* TOS = op(TOS, x[imm]) */
    FI_BIN_P = 5,      /* TOS = op(TOS, c[imm]) */
    FI_HALT = 6
};

struct FIns {
    uint8_t kind;
    uint8_t op;
    uint8_t arg;   /* spill slot of the left operand (FI_BIN_S) */
    uint8_t spill; /* slot a push spills TOS to, 0xff when the stack was empty */
    uint16_t imm;  /* input column or constant slot */
    uint16_t tape; /* first partial-tape slot of this instruction */
};
static_assert(sizeof(FIns) == 8, "FIns is 8 bytes");

/* Partials an operator keeps for the reverse sweep: none for linear ones. */
__host__ __device__ inline int fi_npartials(unsigned op, bool binary)
{
    if (op == OP_ADD || op == OP_SUB || op == OP_NEG) return 0;
    return binary ? 2 : 1;
}

/* Host translation of one fit-record program. Returns false when the records
   are not a tree in stack (post-) order, which the device path rejects. */
inline bool fi_decode(const uint32_t *rec, int m, std::vector<FIns> &out, int *nslots, int *ntape)
{
    std::vector<int> stack;
    int depth = 0, maxslot = -1, tape = 0;
    out.clear();
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
            stack.push_back(i);
            out.push_back(in);
        } else if (ft_op_binary(op)) {
            if (stack.size() < 2 || stack[stack.size() - 1] != (int)k1 ||
                stack[stack.size() - 2] != (int)k0)
                return false;
            stack.pop_back();
            stack.back() = i;
            in.kind = FI_BIN_S;
            in.arg = (uint8_t)(depth - 2);
            --depth;
            const int np = fi_npartials(op, true);
            FIns &prev = out.back();
            if ((prev.kind == FI_PUSH_VAR || prev.kind == FI_PUSH_PARAM) && prev.spill == in.arg) {
                /* fuse "push right operand; op" */
                prev.kind = prev.kind == FI_PUSH_VAR ? FI_BIN_V : FI_BIN_P;
                prev.op = (uint8_t)op;
                prev.spill = 0xff;
                prev.tape = (uint16_t)tape;
            } else {
                out.push_back(in);
            }
            tape += np;
        } else {
            if (stack.empty() || stack.back() != (int)k0) return false;
            stack.back() = i;
            in.kind = FI_UNARY;
            tape += fi_npartials(op, false);
            out.push_back(in);
        }
    }
    if (stack.size() != 1 || stack[0] != m - 1) return false;
    FIns h;
    h.kind = FI_HALT;
    h.op = 0;
    h.arg = 0;
    h.spill = 0xff;
    h.imm = 0;
    h.tape = (uint16_t)tape;
    out.push_back(h);
    *nslots = maxslot + 1;
    *ntape = tape;
    return true;
}

/* f32 local partials of one operator (ft_partials_f semantics). A `pow`
   with a non-positive base passes nothing. */
__device__ __forceinline__ void fi_partials(unsigned op, float x, float y, float r, float &d0,
                                            float &d1)
{
    d0 = 0.0f;
    d1 = 0.0f;
    switch (op) {
        case OP_EXP: d0 = r; break;
        case OP_LOG: d0 = 1.0f / x; break;
        case OP_ABS: d0 = x >= 0.0f ? 1.0f : -1.0f; break;
        case OP_SQRT: d0 = 1.0f / (2.0f * r); break;
        case OP_SIN: d0 = cosf(x); break;
        case OP_COS: d0 = -sinf(x); break;
        case OP_TAN: {
            const float t = cosf(x);
            d0 = 1.0f / (t * t);
        } break;
        case OP_SINH: d0 = coshf(x); break;
        case OP_COSH: d0 = sinhf(x); break;
        case OP_TANH: d0 = 1.0f - r * r; break;
        case OP_SIG: d0 = r * (1.0f - r); break;
        case OP_GAUSS: d0 = (-2.0f * x) * r; break;
        case OP_SQUARE: d0 = 2.0f * x; break;
        case OP_CUBE: d0 = 3.0f * x * x; break;
        case OP_ERF: d0 = 1.1283791670955126f * expf(-x * x); break;
        case OP_ERFC: d0 = -1.1283791670955126f * expf(-x * x); break;
        case OP_MUL: d0 = y; d1 = x; break;
        case OP_DIV: d0 = 1.0f / y; d1 = -x / (y * y); break;
        case OP_POW:
            if (x > 0.0f) {
                d0 = y * powf(x, y - 1.0f);
                d1 = r * logf(x);
            }
            break;
        default: break;
    }
}

__device__ __forceinline__ float fi_child(float a, float d) { return a == 0.0f ? 0.0f : a * d; }

/* Forward sweep of four rows. Constants from `cf`, inputs from the columns
   at `row` (16-byte aligned). With PARTIALS, every non-linear operator stores
   its partials in `tape` ([slot][T] float4). */
template <int T, bool PARTIALS>
__device__ __forceinline__ float4 fi_forward(const FIns *__restrict__ prog, const float *cf,
                                             const float *__restrict__ cols, int npad, int row,
                                             float4 *stk, float4 *tape, int tid)
{
    float t0 = 0.f, t1 = 0.f, t2 = 0.f, t3 = 0.f;
    for (int pc = 0; pc < 512; ++pc) {
        const FIns in = prog[pc];
        const unsigned kind = in.kind;
        if (kind <= FI_PUSH_PARAM) {
            if (in.spill != 0xff) stk[in.spill * T + tid] = make_float4(t0, t1, t2, t3);
            if (kind == FI_PUSH_VAR) {
                const float4 x = __ldg(reinterpret_cast<const float4 *>(
                    cols + (size_t)in.imm * (size_t)npad + row));
                t0 = x.x; t1 = x.y; t2 = x.z; t3 = x.w;
            } else {
                const float c = cf[in.imm];
                t0 = c; t1 = c; t2 = c; t3 = c;
            }
            continue;
        }
        if (kind == FI_UNARY) {
            const float r0 = ft_value_f(in.op, t0, 0.f), r1 = ft_value_f(in.op, t1, 0.f);
            const float r2 = ft_value_f(in.op, t2, 0.f), r3 = ft_value_f(in.op, t3, 0.f);
            if (PARTIALS && in.op != OP_NEG) {
                float d, z;
                float4 dd;
                fi_partials(in.op, t0, 0.f, r0, d, z); dd.x = d;
                fi_partials(in.op, t1, 0.f, r1, d, z); dd.y = d;
                fi_partials(in.op, t2, 0.f, r2, d, z); dd.z = d;
                fi_partials(in.op, t3, 0.f, r3, d, z); dd.w = d;
                tape[in.tape * T + tid] = dd;
            }
            t0 = r0; t1 = r1; t2 = r2; t3 = r3;
            continue;
        }
        if (kind <= FI_BIN_P) {
            float a0, a1, a2, a3, b0, b1, b2, b3;
            if (kind == FI_BIN_S) {
                const float4 a = stk[in.arg * T + tid];
                a0 = a.x; a1 = a.y; a2 = a.z; a3 = a.w;
                b0 = t0; b1 = t1; b2 = t2; b3 = t3;
            } else {
                a0 = t0; a1 = t1; a2 = t2; a3 = t3;
                if (kind == FI_BIN_V) {
                    const float4 x = __ldg(reinterpret_cast<const float4 *>(
                        cols + (size_t)in.imm * (size_t)npad + row));
                    b0 = x.x; b1 = x.y; b2 = x.z; b3 = x.w;
                } else {
                    const float c = cf[in.imm];
                    b0 = c; b1 = c; b2 = c; b3 = c;
                }
            }
            const float r0 = ft_value_f(in.op, a0, b0), r1 = ft_value_f(in.op, a1, b1);
            const float r2 = ft_value_f(in.op, a2, b2), r3 = ft_value_f(in.op, a3, b3);
            if (PARTIALS && in.op != OP_ADD && in.op != OP_SUB) {
                float4 p0, p1;
                fi_partials(in.op, a0, b0, r0, p0.x, p1.x);
                fi_partials(in.op, a1, b1, r1, p0.y, p1.y);
                fi_partials(in.op, a2, b2, r2, p0.z, p1.z);
                fi_partials(in.op, a3, b3, r3, p0.w, p1.w);
                tape[in.tape * T + tid] = p0;
                tape[(in.tape + 1) * T + tid] = p1;
            }
            t0 = r0; t1 = r1; t2 = r2; t3 = r3;
            continue;
        }
        break; /* FI_HALT */
    }
    return make_float4(t0, t1, t2, t3);
}

/* Reverse sweep of four rows (the instructions of `prog`, `nins` of them
   including HALT). Constant adjoints are accumulated into g[i * gs + slot]
   (f32) for row i of the thread: `g` points at the thread's first row. */
template <int T>
__device__ __forceinline__ void fi_reverse(const FIns *__restrict__ prog, int nins, float4 *stk,
                                           const float4 *tape, float *g, int gs, int tid)
{
    float a0 = 1.f, a1 = 1.f, a2 = 1.f, a3 = 1.f;
    float *g0 = g;
    for (int pc = nins - 2; pc >= 0; --pc) {
        const FIns in = prog[pc];
        const unsigned kind = in.kind;
        if (kind <= FI_PUSH_PARAM) {
            if (kind == FI_PUSH_PARAM) {
                g0[in.imm] += a0;
                g0[gs + in.imm] += a1;
                g0[2 * gs + in.imm] += a2;
                g0[3 * gs + in.imm] += a3;
            }
            if (in.spill != 0xff) {
                const float4 s = stk[in.spill * T + tid];
                a0 = s.x; a1 = s.y; a2 = s.z; a3 = s.w;
            }
            continue;
        }
        if (kind == FI_UNARY) {
            if (in.op == OP_NEG) {
                a0 = -a0; a1 = -a1; a2 = -a2; a3 = -a3;
            } else {
                const float4 d = tape[in.tape * T + tid];
                a0 = fi_child(a0, d.x); a1 = fi_child(a1, d.y);
                a2 = fi_child(a2, d.z); a3 = fi_child(a3, d.w);
            }
            continue;
        }
        /* binary: left adjoint (x) and right adjoint (y) */
        float l0, l1, l2, l3, r0, r1, r2, r3;
        if (in.op == OP_ADD) {
            l0 = a0; l1 = a1; l2 = a2; l3 = a3;
            r0 = a0; r1 = a1; r2 = a2; r3 = a3;
        } else if (in.op == OP_SUB) {
            l0 = a0; l1 = a1; l2 = a2; l3 = a3;
            r0 = -a0; r1 = -a1; r2 = -a2; r3 = -a3;
        } else {
            const float4 p0 = tape[in.tape * T + tid];
            const float4 p1 = tape[(in.tape + 1) * T + tid];
            l0 = fi_child(a0, p0.x); l1 = fi_child(a1, p0.y);
            l2 = fi_child(a2, p0.z); l3 = fi_child(a3, p0.w);
            r0 = fi_child(a0, p1.x); r1 = fi_child(a1, p1.y);
            r2 = fi_child(a2, p1.z); r3 = fi_child(a3, p1.w);
        }
        if (kind == FI_BIN_S) {
            /* the left operand's adjoint waits in its spill slot; the right
               operand's subtree is next */
            stk[in.arg * T + tid] = make_float4(l0, l1, l2, l3);
            a0 = r0; a1 = r1; a2 = r2; a3 = r3;
        } else {
            if (kind == FI_BIN_P) {
                g0[in.imm] += r0;
                g0[gs + in.imm] += r1;
                g0[2 * gs + in.imm] += r2;
                g0[3 * gs + in.imm] += r3;
            }
            a0 = l0; a1 = l1; a2 = l2; a3 = l3;
        }
    }
}
