/*
 * The "example" debugging equation (pysweep/equations/example.py:13-26) as a
 * step hook: every variable of the cell gains 1 per level (SCHEME = 1), or,
 * in the two-stage form, 1 at the first stage and 2 over the level before it
 * at the second.  It reads no neighbour, only the cell's own variables
 * (idx + v*VARS) and the previous level (idx - TIMES).
 */
__device__ __constant__ double DT;
__device__ __constant__ double DX;
__device__ __constant__ double DY;
__device__ __constant__ int SCHEME;

__device__ void step(double *s, int idx, int globalTimeStep)
{
    const bool full = globalTimeStep % 2 == 0;
    for (int v = 0; v < NV; ++v) {
        const int i = idx + v * VARS;
        if (SCHEME)
            s[i + TIMES] = s[i] + 1;
        else
            s[i + TIMES] = s[i - (full ? TIMES : 0)] + (full ? 2 : 1);
    }
}
