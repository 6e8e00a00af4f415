// es_taps.cuh -- generated by gen_es_taps.py; do not edit.
// Exponential-of-semicircle kernel (W = 8, beta = 2.3 W): with t = s - 1/2 for the
// fractional grid offset s, tap i (0..3) weighs P_i(t) and tap 7-i weighs P_i(-t),
// P_i(t) = sum_n kEsEven[i][n] t^(2n) + t sum_n kEsOdd[i][n] t^(2n).  Fit error 1.9e-08.
#pragma once

namespace mmn {

constexpr int kEsEvenTerms = 5, kEsOddTerms = 4;
__constant__ float kEsEven[4][5] = {
    {7.544255641e-05f, 2.225094941e-03f, 5.299292039e-03f, 1.492409152e-03f, -2.708597458e-04f},
    {1.765909046e-02f, 9.841921926e-02f, 2.136478946e-02f, -7.556576282e-03f, 7.268397021e-04f},
    {2.611282766e-01f, 2.636119127e-01f, -9.580532461e-02f, 1.367981825e-02f, -9.935779963e-04f},
    {8.656142354e-01f, -3.642575145e-01f, 6.914851069e-02f, -7.617705502e-03f, 4.913107841e-04f},
};
__constant__ float kEsOdd[4][4] = {
    {-6.272384780e-04f, -4.403749947e-03f, -3.884068225e-03f, 3.791726340e-05f},
    {-6.503747404e-02f, -7.388940454e-02f, 7.444368675e-03f, 1.109657809e-03f},
    {-4.859053791e-01f, 4.973948374e-02f, 1.650717109e-02f, -4.649308510e-03f},
    {-5.016627312e-01f, 2.510846555e-01f, -5.972506851e-02f, 8.540749550e-03f},
};

}  // namespace mmn
