// Host build of the device-side allele-frequency fit (kg_alleleN.cuh), for
// the CPU test that compares it with the oracle.  Reads, per site, the allele
// count A, the genotype-class counts (A (A + 1) / 2 of them), the iteration
// cap and maf; prints the fitted frequencies.
#include <cstdio>

#include "kg_alleleN.cuh"

int main() {
    int n = 0;
    if (std::scanf("%d", &n) != 1) return 1;
    for (int v = 0; v < n; v++) {
        kg::AlleleClasses C;
        unsigned long long iters = 0;
        double maf = 0.0;
        if (std::scanf("%d", &C.a) != 1) return 1;
        const int ng = C.a * (C.a + 1) / 2;
        C.n = 0;
        for (int g = 0; g < ng; g++) {
            long long c = 0;
            if (std::scanf("%lld", &c) != 1) return 1;
            if (c > 0) {
                C.cls[C.n] = g;
                C.w[C.n] = (double)c;
                C.n++;
            }
        }
        if (std::scanf("%llu %lf", &iters, &maf) != 2) return 1;
        double f[kg::MAXA];
        kg::allele_fit(C, iters, maf, f);
        std::printf("%.17g %.17g %.17g %.17g\n", f[0], f[1], f[2], f[3]);
    }
    return 0;
}
