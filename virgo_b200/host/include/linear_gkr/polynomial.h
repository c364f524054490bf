// Univariate sumcheck message types with the reference's layout and names
// (include/linear_gkr/polynomial.h): coefficients highest degree first.
#ifndef __polynomial
#define __polynomial
#include <vector>
#include "linear_gkr/prime_field.h"

class linear_poly;

// f(x) = a x^3 + b x^2 + c x + d
class cubic_poly
{
public:
    prime_field::field_element a, b, c, d;
    cubic_poly();
    cubic_poly(const prime_field::field_element &, const prime_field::field_element &, const prime_field::field_element &,
               const prime_field::field_element &);
    cubic_poly operator+(const cubic_poly &) const;
    prime_field::field_element eval(const prime_field::field_element &) const;
};

// f(x) = a x^2 + b x + c
class quadratic_poly
{
public:
    prime_field::field_element a, b, c;
    quadratic_poly();
    quadratic_poly(const prime_field::field_element &, const prime_field::field_element &, const prime_field::field_element &);
    quadratic_poly operator+(const quadratic_poly &) const;
    cubic_poly operator*(const linear_poly &) const;
    prime_field::field_element eval(const prime_field::field_element &) const;
};

// f(x) = a x + b
class linear_poly
{
public:
    prime_field::field_element a, b;
    linear_poly();
    linear_poly(const prime_field::field_element &, const prime_field::field_element &);
    linear_poly(const prime_field::field_element &);
    linear_poly operator+(const linear_poly &) const;
    quadratic_poly operator*(const linear_poly &) const;
    prime_field::field_element eval(const prime_field::field_element &) const;
};

// f(x) = a x^4 + b x^3 + c x^2 + d x + e
class quadruple_poly
{
public:
    prime_field::field_element a, b, c, d, e;
    quadruple_poly();
    quadruple_poly(const prime_field::field_element &, const prime_field::field_element &, const prime_field::field_element &,
                   const prime_field::field_element &, const prime_field::field_element &);
    quadruple_poly operator+(const quadruple_poly &) const;
    prime_field::field_element eval(const prime_field::field_element &) const;
};

// f(x) = a x^5 + b x^4 + c x^3 + d x^2 + e x + f
class quintuple_poly
{
public:
    prime_field::field_element a, b, c, d, e, f;
    quintuple_poly();
    quintuple_poly(const prime_field::field_element &, const prime_field::field_element &, const prime_field::field_element &,
                   const prime_field::field_element &, const prime_field::field_element &, const prime_field::field_element &);
    quintuple_poly operator+(const quintuple_poly &) const;
    prime_field::field_element eval(const prime_field::field_element &) const;
};

#endif
