// HVM-64 numbers (the OPER / MATCH payloads), shared by host and device code.
//
// A Num is 32 bits: payload << 8 | tag << 3 | 3 (num/src/num.rs:10-63).  The
// tag is a type (u24, i24, f24), the "symbol" tag, or an operator; an
// operator-tagged Num holds a partially applied operand.  All arithmetic
// follows num/src/num.rs:133-263 bit for bit: integer ops wrap, shift
// amounts are masked to 5 bits (Rust wrapping_shl/shr), f24 is an f32 with
// its low 8 bits rounded off to nearest-even, and float ops are single IEEE
// operations with no contraction (device code is built with -fmad=false and
// uses explicitly rounded intrinsics).  Integer division by zero, which
// panics in the reference, reports HVM64_ERR_DIV0 through `err`.
#pragma once
#include <stdint.h>
#include <string.h>
#include <math.h>

#ifdef __CUDACC__
#define HVM_HD __host__ __device__ __forceinline__
#else
#define HVM_HD inline
#endif

namespace hvm {

enum NumTag : uint8_t {
  NT_U24 = 0, NT_I24, NT_F24, NT_SYM, NT_ADD, NT_SUB, NT_SUBS, NT_MUL, NT_DIV, NT_DIVS,
  NT_REM, NT_REMS, NT_AND, NT_OR, NT_XOR, NT_SHL, NT_SHLS, NT_SHR, NT_SHRS, NT_EQ, NT_NE,
  NT_LT, NT_GT, NT_COUNT
};

HVM_HD uint32_t num_make(uint32_t tag, uint32_t payload) { return (payload << 8) | (tag << 3) | 3u; }
HVM_HD uint32_t num_u24(uint32_t v) { return num_make(NT_U24, v); }
HVM_HD uint32_t num_i24(int32_t v) { return num_make(NT_I24, (uint32_t)v); }
HVM_HD uint32_t num_sym(uint32_t t) { return num_make(NT_SYM, t); }
HVM_HD uint32_t num_invalid() { return num_u24(0); }
HVM_HD uint32_t num_tag(uint32_t n) { return (n >> 3) & 0x1f; }
HVM_HD uint32_t num_payload(uint32_t n) { return n >> 8; }
HVM_HD int32_t num_get_i24(uint32_t n) { return ((int32_t)n) >> 8; }
HVM_HD bool tag_is_op(uint32_t t) { return t > NT_SYM; }

HVM_HD uint32_t f32_bits(float f) {
#ifdef __CUDA_ARCH__
  return __float_as_uint(f);
#else
  uint32_t b;
  memcpy(&b, &f, 4);
  return b;
#endif
}
HVM_HD float bits_f32(uint32_t b) {
#ifdef __CUDA_ARCH__
  return __uint_as_float(b);
#else
  float f;
  memcpy(&f, &b, 4);
  return f;
#endif
}
HVM_HD bool f32_isnan(float f) { return (f32_bits(f) & 0x7fffffffu) > 0x7f800000u; }
HVM_HD float num_get_f24(uint32_t n) { return bits_f32(n & ~0xffu); }

// num.rs:81-90: drop the low byte rounding to nearest-even; NaN stays NaN.
HVM_HD uint32_t num_f24(float val) {
  uint32_t bits = f32_bits(val);
  uint32_t shifted = bits >> 8;
  uint32_t lost = bits & 0xFFu;
  uint32_t nan = f32_isnan(val) ? 1u : 0u;
  shifted += (nan ^ 1u) & ((lost - ((lost >> 7) & ~shifted)) >> 7);
  shifted |= nan;
  return num_make(NT_F24, shifted);
}

// Rust `f as u32` / `f as i32`: round toward zero, saturate, NaN -> 0.
HVM_HD uint32_t sat_u32(float f) {
  if (f32_isnan(f) || f <= 0.0f) return 0;
  if (f >= 4294967296.0f) return 0xFFFFFFFFu;
  return (uint32_t)f;
}
HVM_HD int32_t sat_i32(float f) {
  if (f32_isnan(f)) return 0;
  if (f <= -2147483648.0f) return INT32_MIN;
  if (f >= 2147483648.0f) return INT32_MAX;
  return (int32_t)f;
}

HVM_HD float f_add(float a, float b) {
#ifdef __CUDA_ARCH__
  return __fadd_rn(a, b);
#else
  return a + b;
#endif
}
HVM_HD float f_sub(float a, float b) {
#ifdef __CUDA_ARCH__
  return __fsub_rn(a, b);
#else
  return a - b;
#endif
}
HVM_HD float f_mul(float a, float b) {
#ifdef __CUDA_ARCH__
  return __fmul_rn(a, b);
#else
  return a * b;
#endif
}
HVM_HD float f_div(float a, float b) {
#ifdef __CUDA_ARCH__
  return __fdiv_rn(a, b);
#else
  return a / b;
#endif
}

// num.rs:133-161
HVM_HD uint32_t num_unary(uint32_t op, uint32_t num) {
  const uint32_t U24_MAX = (1u << 24) - 1;
  const int32_t I24_MAX = (1 << 23) - 1, I24_MIN = -(1 << 23);
  uint32_t t = num_tag(num);
  switch (op) {
    case NT_SYM: return num;
    case NT_U24:
      if (t == NT_U24) return num;
      if (t == NT_I24) return num_u24(num_payload(num));
      if (t == NT_F24) {
        uint32_t v = sat_u32(num_get_f24(num));
        return num_u24(v < U24_MAX ? v : U24_MAX);
      }
      return num_invalid();
    case NT_I24:
      if (t == NT_U24) return num_i24(num_get_i24(num));
      if (t == NT_I24) return num;
      if (t == NT_F24) {
        int32_t v = sat_i32(num_get_f24(num));
        v = v < I24_MIN ? I24_MIN : (v > I24_MAX ? I24_MAX : v);
        return num_i24(v);
      }
      return num_invalid();
    case NT_F24:
      if (t == NT_U24) return num_f24((float)num_payload(num));
      if (t == NT_I24) return num_f24((float)num_get_i24(num));
      if (t == NT_F24) return num;
      return num_invalid();
    default: return num_make(op, num_payload(num));
  }
}

// num.rs:164-254.  After the symmetric match, `a` is the operator-tagged
// operand and `b` the typed one.
HVM_HD uint32_t num_sym_op(uint32_t a, uint32_t b, int* err) {
  uint32_t at = num_tag(a), bt = num_tag(b);
  if (at == NT_SYM && bt == NT_SYM) return num_invalid();
  if (at == NT_SYM) return num_unary(num_payload(a) & 0xff, b);
  if (bt == NT_SYM) return num_unary(num_payload(b) & 0xff, a);
  bool ao = tag_is_op(at), bo = tag_is_op(bt);
  if (ao == bo) return num_invalid();
  uint32_t op, ty;
  if (ao) { op = at; ty = bt; } else { op = bt; ty = at; uint32_t s = a; a = b; b = s; }
  if (ty == NT_U24) {
    uint32_t x = num_payload(a), y = num_payload(b);
    switch (op) {
      case NT_ADD: return num_u24(x + y);
      case NT_SUB: return num_u24(x - y);
      case NT_SUBS: return num_u24(y - x);
      case NT_MUL: return num_u24(x * y);
      case NT_DIV: if (y == 0) { *err = 1; return num_invalid(); } return num_u24(x / y);
      case NT_DIVS: if (x == 0) { *err = 1; return num_invalid(); } return num_u24(y / x);
      case NT_REM: if (y == 0) { *err = 1; return num_invalid(); } return num_u24(x % y);
      case NT_REMS: if (x == 0) { *err = 1; return num_invalid(); } return num_u24(y % x);
      case NT_EQ: return num_u24(x == y);
      case NT_NE: return num_u24(x != y);
      case NT_LT: return num_u24(x < y);
      case NT_GT: return num_u24(x > y);
      case NT_AND: return num_u24(x & y);
      case NT_OR: return num_u24(x | y);
      case NT_XOR: return num_u24(x ^ y);
      case NT_SHL: return num_u24(x << (y & 31));
      case NT_SHLS: return num_u24(y << (x & 31));
      case NT_SHR: return num_u24(x >> (y & 31));
      case NT_SHRS: return num_u24(y >> (x & 31));
      default: return num_invalid();
    }
  }
  if (ty == NT_I24) {
    int32_t x = num_get_i24(a), y = num_get_i24(b);
    switch (op) {
      case NT_ADD: return num_i24((int32_t)((uint32_t)x + (uint32_t)y));
      case NT_SUB: return num_i24((int32_t)((uint32_t)x - (uint32_t)y));
      case NT_SUBS: return num_i24((int32_t)((uint32_t)y - (uint32_t)x));
      case NT_MUL: return num_i24((int32_t)((uint32_t)x * (uint32_t)y));
      case NT_DIV:
        if (y == 0) { *err = 1; return num_invalid(); }
        return num_i24((x == INT32_MIN && y == -1) ? x : x / y);
      case NT_DIVS:
        if (x == 0) { *err = 1; return num_invalid(); }
        return num_i24((y == INT32_MIN && x == -1) ? y : y / x);
      case NT_REM:
        if (y == 0) { *err = 1; return num_invalid(); }
        return num_i24(y == -1 ? 0 : x % y);
      case NT_REMS:
        if (x == 0) { *err = 1; return num_invalid(); }
        return num_i24(x == -1 ? 0 : y % x);
      case NT_EQ: return num_u24(x == y);
      case NT_NE: return num_u24(x != y);
      case NT_LT: return num_u24(x < y);
      case NT_GT: return num_u24(x > y);
      case NT_AND: return num_i24(x & y);
      case NT_OR: return num_i24(x | y);
      case NT_XOR: return num_i24(x ^ y);
      case NT_SHL: return num_i24((int32_t)((uint32_t)x << ((uint32_t)y & 31)));
      case NT_SHLS: return num_i24((int32_t)((uint32_t)y << ((uint32_t)x & 31)));
      case NT_SHR: return num_i24(x >> ((uint32_t)y & 31));
      case NT_SHRS: return num_i24(y >> ((uint32_t)x & 31));
      default: return num_invalid();
    }
  }
  if (ty == NT_F24) {
    float x = num_get_f24(a), y = num_get_f24(b);
    switch (op) {
      case NT_ADD: return num_f24(f_add(x, y));
      case NT_SUB: return num_f24(f_sub(x, y));
      case NT_SUBS: return num_f24(f_sub(y, x));
      case NT_MUL: return num_f24(f_mul(x, y));
      case NT_DIV: return num_f24(f_div(x, y));
      case NT_DIVS: return num_f24(f_div(y, x));
      case NT_REM: return num_f24(fmodf(x, y));
      case NT_REMS: return num_f24(fmodf(y, x));
      case NT_EQ: return num_u24(x == y);
      case NT_NE: return num_u24(x != y);
      case NT_LT: return num_u24(x < y);
      case NT_GT: return num_u24(x > y);
      // f24 `&`, `|`, `^` are atan2, log base, pow (num.rs:243-248); their
      // last-bit results follow the platform's libm, which no reference test
      // pins.
      case NT_AND: return num_f24(atan2f(x, y));
      case NT_OR: return num_f24(f_div(logf(y), logf(x)));
      case NT_XOR: return num_f24(powf(x, y));
      default: return num_invalid();
    }
  }
  return num_invalid();
}

// num.rs:257-263
HVM_HD uint32_t num_binary(uint32_t a, uint32_t op, uint32_t b, int* err) {
  if (op == NT_SYM) return num_sym_op(a, b, err);
  return num_sym_op(num_sym_op(a, num_sym(op), err), b, err);
}

}  // namespace hvm
