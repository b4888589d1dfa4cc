// fmvd_deconvolve command-line tool: same flags as the reference CLI
// (fmvd_deconvolve_hdd.cpp:22-180): raw views in, raw result out, through
// fmvd_deconvolve_files_cuda_16 / _8.
//
//   fmvd_deconvolve -v <nViews> -i <iterations> -t <psf type> -o <output>
//                   -d <view files...> -w <weight files...> -k <kernel files...>
//                   -dw <w> -dh <h> -dd <d> -kw <kw> -kh <kh> [-8bit]
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fmvd_deconvolve.h"

static void usage()
{
    printf("Usage:\n");
    printf("fmvd_deconvolve -v <nViews>\n");
    printf("                -i <nIterations>\n");
    printf("                -t <iteration type>\n");
    printf("                -o <output file>\n");
    printf("                -d <datafile view1> <datafile view2> ...\n");
    printf("                -w <weightfile view1> <weightfile view2> ...\n");
    printf("                -k <kernelfile view1> <kernelfile view2> ...\n");
    printf("                -dw <data width>\n");
    printf("                -dh <data height>\n");
    printf("                -dd <data depth>\n");
    printf("                -kw <kernel width>\n");
    printf("                -kh <kernel height>\n");
    printf("                [-8bit]\n");
}

static int read_floats(const char *path, float *dst, size_t n)
{
    FILE *f = fopen(path, "rb");
    if (!f) {
        printf("Could not open %s for reading\n", path);
        return -1;
    }
    size_t got = fread(dst, sizeof(float), n, f);
    fclose(f);
    if (got != n) {
        printf("Short read from %s\n", path);
        return -1;
    }
    return 0;
}

int main(int argc, char **argv)
{
    int i = 1;
    if (argc < 3 || strcmp(argv[i++], "-v")) {
        usage();
        return -1;
    }
    int nViews = atoi(argv[i++]);
    if (nViews < 1) {
        usage();
        return -1;
    }
    int nIterations = 0, type = 0, w = 0, h = 0, d = 0, kw = 0, kh = 0, eightbit = 0;
    const char *output = NULL;
    const char **datafiles = (const char **)calloc(nViews, sizeof(char *));
    const char **weightfiles = (const char **)calloc(nViews, sizeof(char *));
    const char **kernelfiles = (const char **)calloc(nViews, sizeof(char *));
    for (; i < argc; i++) {
        const char *a = argv[i];
        const int more = i + 1 < argc;
        if (!strcmp(a, "-i") && more) nIterations = atoi(argv[++i]);
        else if (!strcmp(a, "-t") && more) type = atoi(argv[++i]);
        else if (!strcmp(a, "-dw") && more) w = atoi(argv[++i]);
        else if (!strcmp(a, "-dh") && more) h = atoi(argv[++i]);
        else if (!strcmp(a, "-dd") && more) d = atoi(argv[++i]);
        else if (!strcmp(a, "-kw") && more) kw = atoi(argv[++i]);
        else if (!strcmp(a, "-kh") && more) kh = atoi(argv[++i]);
        else if (!strcmp(a, "-o") && more) output = argv[++i];
        else if (!strcmp(a, "-8bit")) eightbit = 1;
        else if (!strcmp(a, "-d") || !strcmp(a, "-w") || !strcmp(a, "-k")) {
            const char **dst = a[1] == 'd' ? datafiles : (a[1] == 'w' ? weightfiles : kernelfiles);
            for (int v = 0; v < nViews; v++) {
                if (i + 1 >= argc) {
                    usage();
                    return -1;
                }
                dst[v] = argv[++i];
            }
        }
    }
    if (!output || w < 1 || h < 1 || d < 0 || kw < 1 || kh < 1) {
        usage();
        return -1;
    }
    for (int v = 0; v < nViews; v++)
        if (!datafiles[v] || !weightfiles[v] || !kernelfiles[v]) {
            usage();
            return -1;
        }

    printf("Starting plane-wise deconvolution\n");
    printf("\tnViews:        %d\n", nViews);
    printf("\tnIterations:   %d\n", nIterations);
    printf("\titerationType: %d\n", type);
    printf("\tdimensions:    %d x %d x %d\n", w, h, d);
    printf("\tkernel dims:   %d x %d\n", kw, kh);

    float **kernels = (float **)malloc(nViews * sizeof(float *));
    float **weights = (float **)malloc(nViews * sizeof(float *));
    FILE **files = (FILE **)malloc(nViews * sizeof(FILE *));
    for (int v = 0; v < nViews; v++) {
        kernels[v] = (float *)fmvd_malloc((size_t)kw * kh * sizeof(float));
        weights[v] = (float *)malloc((size_t)w * h * sizeof(float));
        if (read_floats(kernelfiles[v], kernels[v], (size_t)kw * kh) || read_floats(weightfiles[v], weights[v], (size_t)w * h))
            return -1;
        files[v] = fopen(datafiles[v], "rb");
        if (!files[v]) {
            printf("Could not open %s for reading\n", datafiles[v]);
            return -1;
        }
    }
    FILE *result = fopen(output, "wb");
    if (!result) {
        printf("Could not open %s for writing\n", output);
        return -1;
    }
    if (eightbit)
        fmvd_deconvolve_files_cuda_8(files, result, w, h, d, weights, kernels, kh, kw, (fmvd_psf_type)type, nViews,
                                     nIterations);
    else
        fmvd_deconvolve_files_cuda_16(files, result, w, h, d, weights, kernels, kh, kw, (fmvd_psf_type)type, nViews,
                                      nIterations);
    for (int v = 0; v < nViews; v++) {
        fclose(files[v]);
        fmvd_free(kernels[v]);
        free(weights[v]);
    }
    fclose(result);
    free(kernels);
    free(weights);
    free(files);
    free(datafiles);
    free(weightfiles);
    free(kernelfiles);
    return 0;
}
