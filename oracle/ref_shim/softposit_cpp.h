/*
 * softposit_cpp.h -- stand-in for SoftPosit's C++ posit32 class, used ONLY to
 * compile the reference's own libRpack CPU sources out of tree into oracle/_ref
 * (SoftPosit itself is an absent third-party dependency).
 *
 *   a + b, a * b     the reference's own p32_add / p32_mul from
 *                    libRpack/kernel_entry.cl:370-538, compiled from the reference tree
 *   a - b            p32_add(a, -b)
 *   a / b, sqrt(a), posit32(double)
 *                    correctly rounded routines of the oracle restatement (no
 *                    reference source exists for them: parity unpinned)
 *   comparisons      signed-integer order of the patterns (NaR lowest)
 *
 * Test infrastructure only: never linked into the product library.
 */
#ifndef ORACLE_REF_SOFTPOSIT_CPP_H
#define ORACLE_REF_SOFTPOSIT_CPP_H
#include <stdint.h>

extern "C" {
uint32_t ref_p32_add(uint32_t a, uint32_t b);
uint32_t ref_p32_mul(uint32_t a, uint32_t b);
uint32_t orc_p32_div(uint32_t a, uint32_t b);
uint32_t orc_p32_sqrt(uint32_t a);
uint32_t orc_p32_from_double(double x);
double orc_p32_to_double(uint32_t a);
}

struct posit32 {
    uint32_t value;
    posit32() : value(0) {}
    posit32(double x) : value(orc_p32_from_double(x)) {}
    posit32(float x) : value(orc_p32_from_double((double)x)) {}
    posit32(int x) : value(orc_p32_from_double((double)x)) {}
    static posit32 bits(uint32_t u) { posit32 p; p.value = u; return p; }

    posit32 operator-() const { return bits(0u - value); }
    posit32 operator+(const posit32 &o) const { return bits(ref_p32_add(value, o.value)); }
    posit32 operator-(const posit32 &o) const { return bits(ref_p32_add(value, 0u - o.value)); }
    posit32 operator*(const posit32 &o) const { return bits(ref_p32_mul(value, o.value)); }
    posit32 operator/(const posit32 &o) const { return bits(orc_p32_div(value, o.value)); }
    posit32 &operator+=(const posit32 &o) { value = ref_p32_add(value, o.value); return *this; }
    posit32 &operator-=(const posit32 &o) { value = ref_p32_add(value, 0u - o.value); return *this; }
    posit32 &operator*=(const posit32 &o) { value = ref_p32_mul(value, o.value); return *this; }
    posit32 &operator/=(const posit32 &o) { value = orc_p32_div(value, o.value); return *this; }
    bool operator==(const posit32 &o) const { return value == o.value; }
    bool operator!=(const posit32 &o) const { return value != o.value; }
    bool operator<(const posit32 &o) const { return (int32_t)value < (int32_t)o.value; }
    bool operator<=(const posit32 &o) const { return (int32_t)value <= (int32_t)o.value; }
    bool operator>(const posit32 &o) const { return (int32_t)value > (int32_t)o.value; }
    bool operator>=(const posit32 &o) const { return (int32_t)value >= (int32_t)o.value; }
    double toDouble() const { return orc_p32_to_double(value); }
};

inline posit32 sqrt(posit32 a) { return posit32::bits(orc_p32_sqrt(a.value)); }

#endif
