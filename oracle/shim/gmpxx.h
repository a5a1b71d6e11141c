/*
 * Declaration-only stand-in for <gmpxx.h> (see gmp.h in this directory).
 * The class types exist so that type lists and overloads in the reference
 * headers compile; no member is defined.
 */
#pragma once
#include "gmp.h"

class mpz_class
{
        mpz_t value_;

public:
        mpz_class();
        mpz_class(long);
        mpz_class(const mpz_class&);
        mpz_class& operator=(const mpz_class&);
        mpz_class& operator=(long);
        ~mpz_class();
        mpz_ptr get_mpz_t();
        mpz_srcptr get_mpz_t() const;
};

bool operator==(const mpz_class&, long);
bool operator!=(const mpz_class&, long);
bool operator<(const mpz_class&, long);
bool operator<=(const mpz_class&, long);
bool operator>(const mpz_class&, long);
bool operator>=(const mpz_class&, long);

class mpq_class
{
        mpz_t num_;
        mpz_t den_;

public:
        mpq_class();
};

class mpf_class
{
        double value_;

public:
        mpf_class();
        mpf_class(double);
        mpf_class(double, unsigned long);
        mpf_class& operator=(const mpz_class&);
        mpf_class& operator/=(const mpf_class&);
        mpf_ptr get_mpf_t();
        mpf_srcptr get_mpf_t() const;
        double get_d() const;
};
