/*
 * Declaration-only stand-in for <gmp.h>, used only to compile the reference
 * painter as a CPU test oracle.  The painter's render path never performs
 * multi-precision arithmetic (the reference's convex hull does, and the
 * oracle's hull library takes hull_gmp/ and the system's libgmp instead), so
 * nothing here has a definition: any accidental use fails at link time
 * instead of computing a wrong value.
 */
#pragma once
#include <cstddef>

struct nbpt_oracle_mpz_struct
{
        int alloc;
        int size;
        void* data;
};
typedef nbpt_oracle_mpz_struct mpz_t[1];
typedef nbpt_oracle_mpz_struct* mpz_ptr;
typedef const nbpt_oracle_mpz_struct* mpz_srcptr;

struct nbpt_oracle_mpf_struct
{
        int prec;
        int size;
        long exp;
        void* data;
};
typedef nbpt_oracle_mpf_struct mpf_t[1];
typedef nbpt_oracle_mpf_struct* mpf_ptr;
typedef const nbpt_oracle_mpf_struct* mpf_srcptr;

int mpz_sgn(mpz_srcptr);
void mpz_gcd(mpz_ptr, mpz_srcptr, mpz_srcptr);
void mpz_divexact(mpz_ptr, mpz_srcptr, mpz_srcptr);
void mpz_addmul(mpz_ptr, mpz_srcptr, mpz_srcptr);
void mpf_sqrt(mpf_ptr, mpf_srcptr);
void mpf_set_z(mpf_ptr, mpz_srcptr);

void mpz_import(mpz_ptr, std::size_t, int, std::size_t, int, std::size_t, const void*);
void mpz_neg(mpz_ptr, mpz_srcptr);
void mpz_mul(mpz_ptr, mpz_srcptr, mpz_srcptr);
void mpz_submul(mpz_ptr, mpz_srcptr, mpz_srcptr);
void mpz_add(mpz_ptr, mpz_srcptr, mpz_srcptr);
void mpz_sub(mpz_ptr, mpz_srcptr, mpz_srcptr);
