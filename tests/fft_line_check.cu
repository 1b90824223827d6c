// Host driver for tests/test_fft_host.py: reads "n sign" and 2n doubles (re,
// im pairs) from stdin, writes the line transform of pygcmc_b200's mesh FFT
// (fft_line_host, the same Stockham stages the kernels run) to stdout.
#include <cstdio>
#include <cmath>
#include "../pygcmc_b200/csrc/fft.cuh"

int main() {
    int n = 0, sign = 0;
    while (std::scanf("%d %d", &n, &sign) == 2) {
        if (!gcmc::fft_size_ok(n)) {
            std::printf("bad\n");
            return 1;
        }
        double2 x[gcmc::kFftMax];
        for (int i = 0; i < n; ++i) std::scanf("%lf %lf", &x[i].x, &x[i].y);
        gcmc::fft_line_host(x, n, sign);
        for (int i = 0; i < n; ++i) std::printf("%.17g %.17g\n", x[i].x, x[i].y);
    }
    return 0;
}
