/*
 * The "half" debugging equation (pysweep/equations/half.py:15-19, 45-49) as a
 * step hook in the reference's plugin format: a two-stage Runge-Kutta step of
 * the Laplacian divided by 100, in the numpy plugin's operation order.
 */
__device__ __constant__ double DT;
__device__ __constant__ double DX;
__device__ __constant__ double DY;

__device__ double central(double *s, int idx)
{
    const double x = (s[idx + SY] - 2 * s[idx] + s[idx - SY]) / 100;
    const double y = (s[idx + 1] - 2 * s[idx] + s[idx - 1]) / 100;
    return x + y;
}

__device__ void step(double *s, int idx, int globalTimeStep)
{
    const bool full = globalTimeStep % 2 == 0;
    const double coeff = full ? 1.0 : 0.5;
    s[idx + TIMES] = s[idx - (full ? TIMES : 0)] + coeff * central(s, idx);
}
