// Host-side preparation done once per mesh: the uniform BUQ mesh (block origins
// and neighbour tables), as the reference builds it at set-up (src/Mesh.cu:257-433).
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <vector>

#include "../../include/bg_flood_b200.h"


extern "C" int bgf_mesh_uniform(int nbx, int nby, double levdx, const uint8_t* present, int* nblk, int* level,
                                int* nbr8, double* xo, double* yo, int doubleprecision)
{
    if (nbx <= 0 || nby <= 0 || !nblk || !level || !nbr8) return BGF_EINVAL;
    // InitBlockxoyo (src/Mesh.cu:257-347): row-major candidate blocks, masked ones skipped.
    std::vector<int> id((size_t)nbx * nby, -1);
    int n = 0;
    for (int by = 0; by < nby; by++)
        for (int bx = 0; bx < nbx; bx++) {
            size_t k = (size_t)by * nbx + bx;
            if (present && !present[k]) continue;
            id[k] = n;
            level[n] = 0;
            // nblkx * blkwidth * levdx + levdx / 2, evaluated in the state precision
            if (doubleprecision) {
                if (xo) xo[n] = bx * 16.0 * levdx + 0.5 * levdx;
                if (yo) yo[n] = by * 16.0 * levdx + 0.5 * levdx;
            } else {
                const float l = (float)levdx;
                if (xo) xo[n] = (double)(bx * 16.0f * l + 0.5f * l);
                if (yo) yo[n] = (double)(by * 16.0f * l + 0.5f * l);
            }
            n++;
        }
    // InitBlockneighbours (src/Mesh.cu:351-433): neighbours by position, self at edges.
    for (int by = 0; by < nby; by++)
        for (int bx = 0; bx < nbx; bx++) {
            int b = id[(size_t)by * nbx + bx];
            if (b < 0) continue;
            int L = bx > 0 ? id[(size_t)by * nbx + bx - 1] : -1;
            int R = bx < nbx - 1 ? id[(size_t)by * nbx + bx + 1] : -1;
            int B = by > 0 ? id[(size_t)(by - 1) * nbx + bx] : -1;
            int T = by < nby - 1 ? id[(size_t)(by + 1) * nbx + bx] : -1;
            if (L < 0) L = b;
            if (R < 0) R = b;
            if (B < 0) B = b;
            if (T < 0) T = b;
            int* q = nbr8 + 8 * b;
            q[0] = L; q[1] = L; q[2] = R; q[3] = R; q[4] = B; q[5] = B; q[6] = T; q[7] = T;
        }
    *nblk = n;
    return BGF_OK;
}
