/*
 * The "checker" debugging equation (pysweep/equations/checker.py:24-44) as a
 * step hook: every variable becomes the mean of its four neighbours, summed
 * in the numpy plugin's order (x + 1, x - 1, y + 1, y - 1) and divided by 4.
 */
__device__ __constant__ double DT;
__device__ __constant__ double DX;
__device__ __constant__ double DY;
__device__ __constant__ int SCHEME;

__device__ void step(double *s, int idx, int globalTimeStep)
{
    for (int v = 0; v < NV; ++v) {
        const int i = idx + v * VARS;
        double t = s[i + SY];
        t += s[i - SY];
        t += s[i + 1];
        t += s[i - 1];
        s[i + TIMES] = t / 4;
    }
}
