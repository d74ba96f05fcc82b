// Pade approximant coefficients b_0..b_m of exp for the degrees the
// scaling-and-squaring algorithms use (src/Tensile/MatrixExponential.cs:50-110):
// r_m(x) = p_m(x) / p_m(-x), p_m(x) = sum_j b_j x^j.
#pragma once

namespace tns {

inline constexpr double kPade3[] = {120, 60, 12, 1};
inline constexpr double kPade5[] = {30240, 15120, 3360, 420, 30, 1};
inline constexpr double kPade7[] = {17297280, 8648640, 1995840, 277200, 25200, 1512, 56, 1};
inline constexpr double kPade9[] = {17643225600.0, 8821612800.0, 2075673600.0, 302702400.0, 30270240.0,
                                    2162160.0,     110880.0,     3960.0,       90.0,        1.0};
inline constexpr double kPade13[] = {64764752532480000.0, 32382376266240000.0, 7771770303897600.0, 1187353796428800.0,
                                     129060195264000.0,   10559470521600.0,    670442572800.0,     33522128640.0,
                                     1323241920.0,        40840800.0,          960960.0,           16380.0,
                                     182.0,               1.0};

inline const double* pade_coefficients(int m) {
    return m == 3 ? kPade3 : m == 5 ? kPade5 : m == 7 ? kPade7 : m == 9 ? kPade9 : kPade13;
}

}  // namespace tns
