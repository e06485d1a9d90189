/*
 * Node-only natural cubic spline behind the einspline stand-in (bspline.h).
 * TEST INFRASTRUCTURE ONLY.
 *
 * For samples f_0..f_{n-1} on a uniform grid of spacing h, the node slopes m_i
 * of the natural cubic spline solve the tridiagonal system
 *     2 m_0 + m_1               = 3 (f_1 - f_0) / h
 *     m_{i-1} + 4 m_i + m_{i+1} = 3 (f_{i+1} - f_{i-1}) / h      (0 < i < n-1)
 *     m_{n-2} + 2 m_{n-1}       = 3 (f_{n-1} - f_{n-2}) / h
 * (continuity of the second derivative of the piecewise cubic Hermite
 * interpolant, with zero second derivative at both ends).  It is solved here by
 * the Thomas algorithm, one grid line at a time.
 */
#include "bspline.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

static void line_slopes(int n, double h, const double *f, long stride, double *m)
{
    std::vector<double> cp(n), dp(n);
    const double s = 3.0 / h;
    double b = 2.0, c = 1.0;
    double r = s * (f[stride] - f[0]);
    cp[0] = c / b;
    dp[0] = r / b;
    for (int i = 1; i < n; ++i) {
        const double a = 1.0;
        b = (i == n - 1) ? 2.0 : 4.0;
        c = (i == n - 1) ? 0.0 : 1.0;
        if (i == n - 1)
            r = s * (f[(long)i * stride] - f[(long)(i - 1) * stride]);
        else
            r = s * (f[(long)(i + 1) * stride] - f[(long)(i - 1) * stride]);
        const double den = b - a * cp[i - 1];
        cp[i] = c / den;
        dp[i] = (r - a * dp[i - 1]) / den;
    }
    m[(long)(n - 1) * stride] = dp[n - 1];
    for (int i = n - 2; i >= 0; --i)
        m[(long)i * stride] = dp[i] - cp[i] * m[(long)(i + 1) * stride];
}

UBspline_3d_d *create_UBspline_3d_d(Ugrid g0, Ugrid g1, Ugrid g2, BCtype_d bc0, BCtype_d bc1,
                                    BCtype_d bc2, double *data)
{
    if (bc0.lCode != NATURAL || bc0.rCode != NATURAL || bc1.lCode != NATURAL ||
        bc1.rCode != NATURAL || bc2.lCode != NATURAL || bc2.rCode != NATURAL) {
        fprintf(stderr, "nodal spline stand-in: only NATURAL boundaries are supported\n");
        abort();
    }
    UBspline_3d_d *s = new UBspline_3d_d;
    const Ugrid g[3] = {g0, g1, g2};
    for (int d = 0; d < 3; ++d) {
        s->n[d] = g[d].num;
        s->start[d] = g[d].start;
        s->delta[d] = (g[d].end - g[d].start) / (double)(g[d].num - 1);
    }
    const long n0 = s->n[0], n1 = s->n[1], n2 = s->n[2];
    const long N = n0 * n1 * n2;
    s->val = new double[N];
    memcpy(s->val, data, sizeof(double) * N);
    for (int d = 0; d < 3; ++d) s->grad[d] = new double[N];
    for (long a = 0; a < n1; ++a)
        for (long b = 0; b < n2; ++b)
            line_slopes((int)n0, s->delta[0], data + a * n2 + b, n1 * n2, s->grad[0] + a * n2 + b);
    for (long a = 0; a < n0; ++a)
        for (long b = 0; b < n2; ++b)
            line_slopes((int)n1, s->delta[1], data + a * n1 * n2 + b, n2,
                        s->grad[1] + a * n1 * n2 + b);
    for (long a = 0; a < n0; ++a)
        for (long b = 0; b < n1; ++b)
            line_slopes((int)n2, s->delta[2], data + (a * n1 + b) * n2, 1,
                        s->grad[2] + (a * n1 + b) * n2);
    return s;
}

static long node_index(const UBspline_3d_d *s, double x0, double x1, double x2)
{
    const double x[3] = {x0, x1, x2};
    long idx[3];
    for (int d = 0; d < 3; ++d) {
        const double u = (x[d] - s->start[d]) / s->delta[d];
        const double r = std::nearbyint(u);
        if (std::fabs(u - r) > 1e-6 || r < 0 || r > s->n[d] - 1) {
            fprintf(stderr, "nodal spline stand-in: off-node evaluation (axis %d, u=%.17g)\n", d, u);
            abort();
        }
        idx[d] = (long)r;
    }
    return (idx[0] * s->n[1] + idx[1]) * s->n[2] + idx[2];
}

void eval_UBspline_3d_d(UBspline_3d_d *s, double x0, double x1, double x2, double *val)
{
    *val = s->val[node_index(s, x0, x1, x2)];
}

void eval_UBspline_3d_d_vg(UBspline_3d_d *s, double x0, double x1, double x2, double *val,
                           double *grad)
{
    const long i = node_index(s, x0, x1, x2);
    *val = s->val[i];
    grad[0] = s->grad[0][i];
    grad[1] = s->grad[1][i];
    grad[2] = s->grad[2][i];
}

void destroy_Bspline(void *p)
{
    UBspline_3d_d *s = (UBspline_3d_d *)p;
    if (!s) return;
    delete[] s->val;
    for (int d = 0; d < 3; ++d) delete[] s->grad[d];
    delete s;
}
