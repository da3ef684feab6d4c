// Host-side check of the seam kernels' shared-memory layout (swept.cuh):
// the closed-form offsets of the staged faces against brute-force sums, the
// staged area against seam_smem_elems, and the staged / direct choice for
// the shapes the library runs.  Built and run by tests/test_host_layout.py
// (nvcc, no GPU needed).  Prints "ok" or the first mismatch; exit status 0
// on success.
#include <cstdio>

#include "../../pysweep_b200/csrc/swept.cuh"

using psb::seam_direct;
using psb::seam_rows;
using psb::seam_smem_elems;
using psb::seam_xoff;
using psb::seam_yoff;

int main()
{
    for (int gap = 0; gap < 2; ++gap)
        for (int bx : {8, 12, 16, 24, 32, 64})
            for (int ops : {1, 2})
                for (int nv : {1, 4})
                    for (int its : {1, 2}) {
                        const int mpss = bx / (2 * ops) - 1;
                        const int o2 = 2 * ops;
                        for (int hmax = 1; hmax <= mpss; ++hmax) {
                            long ys = 0, xs = 0;
                            for (int m = 1; m <= hmax; ++m) {
                                if (seam_yoff(gap, bx, ops, nv, m) != ys ||
                                    seam_xoff(ops, nv, m) != xs) {
                                    printf("offset mismatch gap %d bx %d ops %d nv %d m %d\n", gap,
                                           bx, ops, nv, m);
                                    return 1;
                                }
                                ys += 2L * nv * seam_rows(gap, bx, ops, m) * o2;
                                xs += (long)nv * 2 * o2 * (2 * ops * m + 2 * o2);
                            }
                            const long slots = (long)(its + 1) * nv * bx * (2 * ops * (hmax + 1));
                            const long total = (long)seam_smem_elems(gap, bx, ops, nv, its, hmax);
                            // the staged area ends where levels 1..hmax-1 end
                            const long want = slots + seam_yoff(gap, bx, ops, nv, hmax) +
                                              (gap ? seam_xoff(ops, nv, hmax) : 0);
                            if (total != want) {
                                printf("size mismatch gap %d bx %d ops %d nv %d hmax %d\n", gap,
                                       bx, ops, nv, hmax);
                                return 1;
                            }
                        }
                    }
    // heat, bs 32, 12 levels: staged (9 CTAs per SM either way);
    // Euler, bs 32, 7 levels: direct (staged would leave one CTA per SM);
    // Euler, bs 16, 3 levels: staged
    if (seam_direct(32, 1, 1, 1, 12, 8) || !seam_direct(32, 2, 4, 2, 7, 8) ||
        seam_direct(16, 2, 4, 2, 3, 8)) {
        printf("staging choice mismatch\n");
        return 1;
    }
    printf("ok\n");
    return 0;
}
