/*
 * Heat equation step hook in the reference's plugin format (the interface of
 * pysweep/equations/heat.cu: __constant__ globals set by name, step() reading
 * neighbours at idx +- SY and idx +- 1 and writing idx + TIMES), with the
 * operation order of the numpy plugin (pysweep/equations/heat.py:48-64), so
 * that its levels equal the reference's CPU levels bit for bit.
 */
__device__ __constant__ double DT;
__device__ __constant__ double DX;
__device__ __constant__ double DY;
__device__ __constant__ double ALPHA;
__device__ __constant__ int SCHEME;  // 1: forward Euler, 0: two-stage Runge-Kutta

__device__ double laplacian(double *s, int idx)
{
    const double courant = ALPHA * DT / DX / DX;
    const double sx = courant * (s[idx + SY] - 2 * s[idx] + s[idx - SY]);
    const double sy = courant * (s[idx + 1] - 2 * s[idx] + s[idx - 1]);
    return sx + sy;
}

__device__ void step(double *s, int idx, int globalTimeStep)
{
    if (SCHEME) {
        s[idx + TIMES] = laplacian(s, idx) + s[idx];
    } else {
        const bool full = globalTimeStep % 2 == 0;  // the second stage rolls back a level
        const double coeff = full ? 1.0 : 0.5;
        s[idx + TIMES] = coeff * laplacian(s, idx) + s[idx - (full ? TIMES : 0)];
    }
}
