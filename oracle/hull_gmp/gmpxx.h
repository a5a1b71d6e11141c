/*
 * A minimal value-semantics mpz_class / mpf_class over GMP's C interface
 * (hull_gmp/gmp.h), with the operations the reference's convex hull and
 * numerical headers apply to them; for the oracle's hull library only.
 * mpq_class exists for the reference's type-name lists and is not usable.
 */
#pragma once
#include "gmp.h"

#include <type_traits>

class mpz_class
{
        mpz_t v_;

public:
        mpz_class()
        {
                __gmpz_init(v_);
        }
        mpz_class(const mpz_class& o)
        {
                __gmpz_init(v_);
                __gmpz_set(v_, o.v_);
        }
        template <typename I>
                requires std::is_integral_v<I>
        mpz_class(const I i)
        {
                __gmpz_init(v_);
                __gmpz_set_si(v_, static_cast<long>(i));
        }
        ~mpz_class()
        {
                __gmpz_clear(v_);
        }
        mpz_class& operator=(const mpz_class& o)
        {
                if (this != &o)
                {
                        __gmpz_set(v_, o.v_);
                }
                return *this;
        }
        template <typename I>
                requires std::is_integral_v<I>
        mpz_class& operator=(const I i)
        {
                __gmpz_set_si(v_, static_cast<long>(i));
                return *this;
        }
        mpz_ptr get_mpz_t()
        {
                return v_;
        }
        mpz_srcptr get_mpz_t() const
        {
                return v_;
        }
        double get_d() const
        {
                return __gmpz_get_d(v_);
        }
        mpz_class& operator+=(const mpz_class& o)
        {
                __gmpz_add(v_, v_, o.v_);
                return *this;
        }
        mpz_class& operator-=(const mpz_class& o)
        {
                __gmpz_sub(v_, v_, o.v_);
                return *this;
        }
        mpz_class& operator*=(const mpz_class& o)
        {
                __gmpz_mul(v_, v_, o.v_);
                return *this;
        }
};

inline mpz_class operator+(const mpz_class& a, const mpz_class& b)
{
        mpz_class r;
        __gmpz_add(r.get_mpz_t(), a.get_mpz_t(), b.get_mpz_t());
        return r;
}
inline mpz_class operator-(const mpz_class& a, const mpz_class& b)
{
        mpz_class r;
        __gmpz_sub(r.get_mpz_t(), a.get_mpz_t(), b.get_mpz_t());
        return r;
}
inline mpz_class operator*(const mpz_class& a, const mpz_class& b)
{
        mpz_class r;
        __gmpz_mul(r.get_mpz_t(), a.get_mpz_t(), b.get_mpz_t());
        return r;
}
inline mpz_class operator-(const mpz_class& a)
{
        mpz_class r;
        __gmpz_neg(r.get_mpz_t(), a.get_mpz_t());
        return r;
}
inline int mpz_compare(const mpz_class& a, const mpz_class& b)
{
        return __gmpz_cmp(a.get_mpz_t(), b.get_mpz_t());
}
inline bool operator==(const mpz_class& a, const mpz_class& b)
{
        return mpz_compare(a, b) == 0;
}
inline bool operator!=(const mpz_class& a, const mpz_class& b)
{
        return mpz_compare(a, b) != 0;
}
inline bool operator<(const mpz_class& a, const mpz_class& b)
{
        return mpz_compare(a, b) < 0;
}
inline bool operator<=(const mpz_class& a, const mpz_class& b)
{
        return mpz_compare(a, b) <= 0;
}
inline bool operator>(const mpz_class& a, const mpz_class& b)
{
        return mpz_compare(a, b) > 0;
}
inline bool operator>=(const mpz_class& a, const mpz_class& b)
{
        return mpz_compare(a, b) >= 0;
}
inline mpz_class abs(const mpz_class& a)
{
        return mpz_sgn(a.get_mpz_t()) < 0 ? -a : a;
}

class mpq_class
{
        int unused_ = 0;
};

class mpf_class
{
        mpf_t v_;

public:
        mpf_class(const double d, const unsigned long precision)
        {
                __gmpf_init2(v_, precision);
                __gmpf_set_d(v_, d);
        }
        mpf_class(const mpf_class& o)
        {
                __gmpf_init2(v_, static_cast<unsigned long>(o.v_->_mp_prec) * 64);
                __gmpf_set(v_, o.v_);
        }
        ~mpf_class()
        {
                __gmpf_clear(v_);
        }
        mpf_class& operator=(const mpf_class& o)
        {
                if (this != &o)
                {
                        __gmpf_set(v_, o.v_);
                }
                return *this;
        }
        mpf_class& operator=(const mpz_class& z)
        {
                __gmpf_set_z(v_, z.get_mpz_t());
                return *this;
        }
        mpf_class& operator/=(const mpf_class& o)
        {
                __gmpf_div(v_, v_, o.v_);
                return *this;
        }
        mpf_ptr get_mpf_t()
        {
                return v_;
        }
        mpf_srcptr get_mpf_t() const
        {
                return v_;
        }
        double get_d() const
        {
                return __gmpf_get_d(v_);
        }
};
