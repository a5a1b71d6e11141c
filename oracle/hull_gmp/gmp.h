/*
 * Declarations of the part of GMP's C interface the reference's convex hull
 * uses, for the oracle's hull library only (oracle/_ref/libnbpt_hull.so),
 * which links the system's libgmp.so.10 (its headers are not installed).
 * The names are GMP's documented ones; the library exports each mpz_X /
 * mpf_X function as __gmpz_X / __gmpf_X.  The structures have GMP's layout.
 */
#pragma once
#include <cstddef>

extern "C" {
typedef unsigned long mp_limb_t;
typedef long mp_exp_t;
typedef unsigned long mp_bitcnt_t;

typedef struct
{
        int _mp_alloc;
        int _mp_size;
        mp_limb_t* _mp_d;
} __mpz_struct;
typedef __mpz_struct mpz_t[1];
typedef __mpz_struct* mpz_ptr;
typedef const __mpz_struct* mpz_srcptr;

typedef struct
{
        int _mp_prec;
        int _mp_size;
        mp_exp_t _mp_exp;
        mp_limb_t* _mp_d;
} __mpf_struct;
typedef __mpf_struct mpf_t[1];
typedef __mpf_struct* mpf_ptr;
typedef const __mpf_struct* mpf_srcptr;

void __gmpz_init(mpz_ptr);
void __gmpz_clear(mpz_ptr);
void __gmpz_set(mpz_ptr, mpz_srcptr);
void __gmpz_set_si(mpz_ptr, long);
void __gmpz_add(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_sub(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_mul(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_neg(mpz_ptr, mpz_srcptr);
void __gmpz_addmul(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_submul(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_gcd(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_divexact(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_import(mpz_ptr, std::size_t, int, std::size_t, int, std::size_t, const void*);
int __gmpz_cmp(mpz_srcptr, mpz_srcptr);
int __gmpz_cmp_si(mpz_srcptr, long);
double __gmpz_get_d(mpz_srcptr);

void __gmpf_init2(mpf_ptr, mp_bitcnt_t);
void __gmpf_clear(mpf_ptr);
void __gmpf_set(mpf_ptr, mpf_srcptr);
void __gmpf_set_d(mpf_ptr, double);
void __gmpf_set_z(mpf_ptr, mpz_srcptr);
void __gmpf_div(mpf_ptr, mpf_srcptr, mpf_srcptr);
void __gmpf_sqrt(mpf_ptr, mpf_srcptr);
double __gmpf_get_d(mpf_srcptr);
}

#define mpz_set __gmpz_set
#define mpz_add __gmpz_add
#define mpz_sub __gmpz_sub
#define mpz_mul __gmpz_mul
#define mpz_neg __gmpz_neg
#define mpz_addmul __gmpz_addmul
#define mpz_submul __gmpz_submul
#define mpz_gcd __gmpz_gcd
#define mpz_divexact __gmpz_divexact
#define mpz_import __gmpz_import
#define mpz_cmp __gmpz_cmp
#define mpf_sqrt __gmpf_sqrt
#define mpf_set_z __gmpf_set_z

inline int mpz_sgn(mpz_srcptr z)
{
        return z->_mp_size < 0 ? -1 : (z->_mp_size > 0 ? 1 : 0);
}
