/*
 * Oracle helper (test infrastructure, never linked into the product).
 *
 * Restates sortBasisArray (module.F90:531-602) exactly: the O(n^2) exchange sort of
 * Basis_type records by (basis(1:nVar) lexicographic, reference), swapping whole records
 * (basis, reference, variation, operation) whenever a(n) > a(m) for m > n.  The sort is
 * not stable: records whose keys tie (same quantum numbers and same reference, which
 * happens when two local operations carry identical quantum numbers) end in the order
 * this exact swap sequence produces, so it is restated swap for swap.
 *
 * rec: n records of (nvar + 3) int32, in the packed order of module.F90:440-466.
 */
#include <stdint.h>
#include <string.h>

static int is_greater(const int32_t *a, const int32_t *b, int nvar)
{
    /* isgreaterBasis, module.F90:549-577 */
    for (int i = 0; i < nvar; ++i) {
        if (a[i] > b[i]) return 1;
        if (a[i] < b[i]) return 0;
    }
    if (a[nvar] > b[nvar]) return 1;
    return 0;
}

void oracle_exchange_sort(int32_t *rec, int64_t n, int nvar)
{
    const int w = nvar + 3;
    int32_t tmp[64];
    for (int64_t i = 0; i < n; ++i) {
        int32_t *a = rec + i * w;
        for (int64_t j = i + 1; j < n; ++j) {
            int32_t *b = rec + j * w;
            if (is_greater(a, b, nvar)) {
                memcpy(tmp, a, sizeof(int32_t) * w);
                memcpy(a, b, sizeof(int32_t) * w);
                memcpy(b, tmp, sizeof(int32_t) * w);
            }
        }
    }
}
