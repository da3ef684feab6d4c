/*
 * A step hook that is not one of the reference's plugins: the linear wave
 * system u_t = -A (v_x + v_y), v_t = -A (u_x + u_y) on two variables, with
 * fourth-order central first derivatives (a five-point stencil per
 * direction, so OPS = 2) and the reference's two-stage Runge-Kutta pattern
 * (the first stage advances half a step from the current level, the second a
 * whole step from the level before it).  Grid spacing 1; A and DT are set by
 * name.
 */
__device__ __constant__ double A;
__device__ __constant__ double DT;

__device__ double d1(double *f, int i, int stride)
{
    return (-f[i + 2 * stride] + 8 * f[i + stride] - 8 * f[i - stride] + f[i - 2 * stride]) / 12;
}

__device__ void step(double *s, int idx, int globalTimeStep)
{
    const bool full = globalTimeStep % ITS == 0;
    const double coeff = full ? 1.0 : 0.5;
    const int back = full ? TIMES : 0;
    const double ru = -A * (d1(s, idx + VARS, SY) + d1(s, idx + VARS, 1));
    const double rv = -A * (d1(s, idx, SY) + d1(s, idx, 1));
    s[idx + TIMES] = s[idx - back] + coeff * DT * ru;
    s[idx + VARS + TIMES] = s[idx + VARS - back] + coeff * DT * rv;
}
