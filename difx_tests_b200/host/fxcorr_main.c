/*
 * fxcorr_main.c -- command-line correlator host over the C ABI (include/fxcorr.h).
 *
 * Reads a .conf file in the reference's grammar (keyword per line, case
 * insensitive: NBIT, COMPLEX, NPOL, NCHAN, LO, BANDWIDTH, NUMFFTS, NANT followed
 * by NANT lines "name file d_quad d_lin d_const fileoffset"; defaults NPOL 2,
 * COMPLEX 0, NBIT 2 -- the grammar of the reference's main.c:14-129), reads one
 * subintegration per antenna file, correlates it on the GPU and writes vis.out
 * in the reference's text format (kernel.c:570-630).  Additional keyword
 * XMODE PLAIN|TC|FP8 selects the X stage; the reference host reports unknown
 * keywords and carries on, so such files stay readable by it.
 *
 * usage: fxcorr_main [config.conf] [-o vis.out] [-b vis.bin] [-x plain|tc|fp8] [-n]
 *   -b  also write all visibilities (crosses then autos) and counts in binary:
 *       int32 header {nsub, nbl+nant, npol*npol, nchan}, counts int32[nbl+nant],
 *       complex float32 [nsub][nbl+nant][npol*npol][nchan]
 *   -n  do not normalise by the baseline counts
 * Exit status: 0 ok, 1 usage/config/IO error, 2 correlator error.
 */
#include <ctype.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>

#include "fxcorr.h"

/* X-stage form by name: TC (FP16 tensor cores), FP8 (E4M3 tensor cores), anything else plain FP32 */
static int parse_xmode(const char* v)
{
    if (!strcasecmp(v, "TC")) return FXC_X_TC_FP16;
    if (!strcasecmp(v, "FP8")) return FXC_X_TC_FP8;
    return FXC_X_PLAIN_FP32;
}

typedef struct {
    int nbit, npol, iscomplex, nchan, nant, numffts, xmode;
    double lo, bw;
    char** names;
    char** files;
    double* delays;      /* [3*ant + k] */
    double* offsets;     /* [ant] */
} conf_t;

static int parse_conf(const char* path, conf_t* c)
{
    FILE* f = fopen(path, "r");
    if (!f) {
        fprintf(stderr, "Error opening file %s\n", path);
        return -1;
    }
    memset(c, 0, sizeof(*c));
    c->npol = 2;
    c->nbit = 2;
    c->xmode = FXC_X_PLAIN_FP32;
    char line[4096];
    int toread = 0, iant = 0, lineno = 0;
    while (fgets(line, sizeof line, f)) {
        lineno++;
        char* tok = strtok(line, " \t\r\n");
        if (!tok) continue;                      /* blank line */
        if (toread) {
            char* file = strtok(NULL, " \t\r\n");
            char* v[4];
            for (int i = 0; i < 4; i++) v[i] = strtok(NULL, " \t\r\n");
            if (!file || !v[0] || !v[1] || !v[2] || !v[3]) {
                fprintf(stderr, "%s:%d: insufficient data for antenna %d\n", path, lineno, iant);
                fclose(f);
                return -1;
            }
            c->names[iant] = strdup(tok);
            c->files[iant] = strdup(file);
            for (int k = 0; k < 3; k++) c->delays[3 * iant + k] = strtod(v[k], NULL);
            c->offsets[iant] = strtod(v[3], NULL);
            iant++;
            toread--;
            continue;
        }
        char* val = strtok(NULL, " \t\r\n");
        if (!strcasecmp(tok, "NANT")) {
            if (!val || (c->nant = atoi(val)) < 2) {
                fprintf(stderr, "%s:%d: bad NANT\n", path, lineno);
                fclose(f);
                return -1;
            }
            c->names = calloc(c->nant, sizeof(char*));
            c->files = calloc(c->nant, sizeof(char*));
            c->delays = calloc(3 * (size_t)c->nant, sizeof(double));
            c->offsets = calloc(c->nant, sizeof(double));
            toread = c->nant;
            iant = 0;
        } else if (!val) {
            fprintf(stderr, "%s:%d: insufficient data for %s\n", path, lineno, tok);
            fclose(f);
            return -1;
        } else if (!strcasecmp(tok, "NBIT")) {
            c->nbit = atoi(val);
        } else if (!strcasecmp(tok, "COMPLEX")) {
            c->iscomplex = atoi(val);
        } else if (!strcasecmp(tok, "NPOL")) {
            c->npol = atoi(val);
        } else if (!strcasecmp(tok, "NCHAN")) {
            c->nchan = atoi(val);
        } else if (!strcasecmp(tok, "LO")) {
            c->lo = strtod(val, NULL);
        } else if (!strcasecmp(tok, "BANDWIDTH")) {
            c->bw = strtod(val, NULL);
        } else if (!strcasecmp(tok, "NUMFFTS")) {
            c->numffts = atoi(val);
        } else if (!strcasecmp(tok, "XMODE")) {
            c->xmode = parse_xmode(val);
        } else {
            fprintf(stderr, "Error: Unknown keyword \"%s\"\n", tok);
        }
    }
    fclose(f);
    if (toread || c->nant < 2 || c->nchan <= 0 || c->numffts <= 0 || c->bw <= 0) {
        fprintf(stderr, "%s: incomplete configuration\n", path);
        return -1;
    }
    return 0;
}

static void write_visout(const char* path, const float* vis, int nbl, int np2, int nchan, double bw)
{
    FILE* f = fopen(path, "w");
    if (!f) {
        fprintf(stderr, "Error opening %s for writing\n", path);
        return;
    }
    for (int c = 0; c < nchan; c++) {
        fprintf(f, "%5d %11.6f", c, (c + 0.5) / nchan * bw / 1e6);
        for (int b = 0; b < nbl; b++)
            for (int p = 0; p < np2; p++) {
                const float re = vis[2 * (((size_t)b * np2 + p) * nchan + c)];
                const float im = vis[2 * (((size_t)b * np2 + p) * nchan + c) + 1];
                fprintf(f, " %11.6f %11.6f", re, im);
                fprintf(f, " %11.6f %10.6f", sqrtf(re * re + im * im), atan2f(im, re));
            }
        fprintf(f, "\n");
    }
    fclose(f);
}

int main(int argc, char** argv)
{
    const char* conf_path = "./test.conf";
    const char* out_path = "vis.out";
    const char* bin_path = NULL;
    int xmode_cli = -1, normalize = 1;
    for (int i = 1; i < argc; i++) {
        if (!strcmp(argv[i], "-o") && i + 1 < argc) out_path = argv[++i];
        else if (!strcmp(argv[i], "-b") && i + 1 < argc) bin_path = argv[++i];
        else if (!strcmp(argv[i], "-x") && i + 1 < argc) {
            i++;
            xmode_cli = parse_xmode(argv[i]);
        } else if (!strcmp(argv[i], "-n")) normalize = 0;
        else if (argv[i][0] != '-') conf_path = argv[i];
        else {
            fprintf(stderr, "usage: %s [config.conf] [-o vis.out] [-b vis.bin] [-x plain|tc|fp8] [-n]\n", argv[0]);
            return 1;
        }
    }
    conf_t c;
    if (parse_conf(conf_path, &c) != 0) return 1;

    fxc_config cfg;
    fxc_config_default(&cfg);
    cfg.nant = c.nant;
    cfg.npol = c.npol;
    cfg.nchan = c.nchan;
    cfg.nbit = c.nbit;
    cfg.iscomplex = c.iscomplex;
    cfg.numffts = c.numffts;
    cfg.lo = c.lo;
    cfg.bw = c.bw;
    cfg.sb_spacing = c.bw;
    cfg.xmode = xmode_cli >= 0 ? xmode_cli : c.xmode;
    const size_t bytes = fxc_subint_bytes(&cfg);

    /* read one subintegration per antenna (openFiles.c / readdata) into pinned memory */
    uint8_t** data = calloc(c.nant, sizeof(uint8_t*));
    for (int a = 0; a < c.nant; a++) {
        void* p = NULL;
        if (fxc_host_alloc(&p, bytes) != FXC_OK) p = malloc(bytes);
        data[a] = p;
        FILE* f = fopen(c.files[a], "rb");
        if (!f) {
            fprintf(stderr, "Problem with file %s - does it exist?\n", c.files[a]);
            return 1;
        }
        const size_t got = fread(data[a], 1, bytes, f);
        fclose(f);
        if (got != bytes) {
            fprintf(stderr, "Error: Problem reading data (Read %zu of %zu bytes from %s)\n", got, bytes, c.files[a]);
            return 1;
        }
    }

    fxc_ctx* ctx = NULL;
    int st = fxc_create(&cfg, &ctx);
    if (st == FXC_OK) st = fxc_process_host(ctx, (const uint8_t* const*)data, c.delays, c.offsets, 0, c.numffts);
    const int nbl = fxc_num_baselines(&cfg);
    const size_t nvis = fxc_vis_count(&cfg);
    float* vis = malloc(2 * sizeof(float) * nvis);
    int* counts = malloc(sizeof(int) * (nbl + c.nant));
    if (st == FXC_OK) st = fxc_get_visibilities(ctx, vis, counts, normalize);
    if (st != FXC_OK) {
        fprintf(stderr, "fxcorr: %s (cuda error %d)\n", fxc_strerror(st), fxc_last_cuda_error());
        return 2;
    }
    write_visout(out_path, vis, nbl, c.npol * c.npol, c.nchan, c.bw);
    if (bin_path) {
        FILE* f = fopen(bin_path, "wb");
        if (f) {
            const int32_t hdr[4] = {1, nbl + c.nant, c.npol * c.npol, c.nchan};
            fwrite(hdr, sizeof hdr, 1, f);
            fwrite(counts, sizeof(int), nbl + c.nant, f);
            fwrite(vis, 2 * sizeof(float), nvis, f);
            fclose(f);
        }
    }
    fxc_destroy(ctx);
    return 0;
}
