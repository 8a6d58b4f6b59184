/*
 * fxcorr_main.c -- command-line correlator host over the C ABI (include/fxcorr.h).
 *
 * Reads a .conf file in the reference's grammar (keyword per line, case
 * insensitive: NBIT, COMPLEX, NPOL, NCHAN, LO, BANDWIDTH, NUMFFTS, NANT followed
 * by NANT lines "name file d_quad d_lin d_const fileoffset"; defaults NPOL 2,
 * COMPLEX 0, NBIT 2 -- the grammar of the reference's main.c:14-129), reads one
 * subintegration per antenna file, correlates it on the GPU and writes vis.out
 * in the reference's text format (kernel.c:570-630).  The reference host reports
 * unknown keywords and carries on, so files with these additional keywords stay
 * readable by it:
 *   XMODE PLAIN|TC|FP8   X-stage form
 *   FSTAGE FFT|TC32|TC16 F-stage arithmetic (fxc_config.fstage; default FFT)
 *   NSUBBAND n           subbands per antenna: the antenna's file name holds one
 *                        printf "%d" replaced by the subband index 0..n-1
 *   SBSPACING hz         LO step between subbands (default BANDWIDTH)
 *   NSUBINT n            successive subintegrations to correlate (default 1)
 *
 * Streaming: subintegration s is the FFTs s*NUMFFTS .. (s+1)*NUMFFTS-1 of each
 * file's continuous sample stream (NUMFFTS+1 FFTs of bytes read, as
 * allocDataHost.c:21 sizes one subintegration), with the delay polynomial
 * shifted to the subintegration's first FFT.  A reader thread fills one pinned
 * buffer set while the GPU correlates the other.
 *
 * usage: fxcorr_main [config.conf] [-o vis.out] [-b vis.bin] [-x plain|tc|fp8] [-f fft|tc32|tc16]
 *                    [-s nsubint] [-n]
 *   -o  text output; with several subintegrations one file per subintegration,
 *       named <out>.<s>
 *   -b  also write all visibilities (crosses then autos) and counts in binary, one
 *       record per subintegration: int32 header {nsubband, nbl+nant, npol*npol,
 *       nchan}, counts int32[nbl+nant], complex float32 [nsubband][nbl+nant][npol*npol][nchan]
 *   -s  successive subintegrations (overrides NSUBINT)
 *   -n  do not normalise by the baseline counts
 * Exit status: 0 ok, 1 usage/config/IO error, 2 correlator error.
 */
#include <ctype.h>
#include <math.h>
#include <pthread.h>
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

/* F-stage arithmetic by name: TC32 (FP32-grade tensor cores), TC16 (FP16 tensor cores),
 * anything else the FP32 FFT */
static int parse_fstage(const char* v)
{
    if (!strcasecmp(v, "TC32")) return FXC_F_TC32;
    if (!strcasecmp(v, "TC16")) return FXC_F_TC16;
    return FXC_F_FFT32;
}

typedef struct {
    int nbit, npol, iscomplex, nchan, nant, numffts, xmode, fstage, nsubband, nsubint;
    double lo, bw, sbspacing;
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
    c->fstage = FXC_F_FFT32;
    c->nsubband = 1;
    c->nsubint = 1;
    c->sbspacing = -1.0;
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
        } else if (!strcasecmp(tok, "FSTAGE")) {
            c->fstage = parse_fstage(val);
        } else if (!strcasecmp(tok, "NSUBBAND")) {
            c->nsubband = atoi(val);
        } else if (!strcasecmp(tok, "SBSPACING")) {
            c->sbspacing = strtod(val, NULL);
        } else if (!strcasecmp(tok, "NSUBINT")) {
            c->nsubint = atoi(val);
        } else {
            fprintf(stderr, "Error: Unknown keyword \"%s\"\n", tok);
        }
    }
    fclose(f);
    if (toread || c->nant < 2 || c->nchan <= 0 || c->numffts <= 0 || c->bw <= 0 || c->nsubband < 1 ||
        c->nsubint < 1) {
        fprintf(stderr, "%s: incomplete configuration\n", path);
        return -1;
    }
    if (c->sbspacing < 0) c->sbspacing = c->bw;
    if (c->nsubband > 1)
        for (int a = 0; a < c->nant; a++) {
            /* the file name is a printf format with exactly one %d (and %% for a literal %) */
            int nd = 0, bad = 0;
            for (const char* q = c->files[a]; *q; q++)
                if (*q == '%') {
                    if (q[1] == '%') q++;
                    else if (q[1] == 'd') nd++, q++;
                    else bad = 1;
                }
            if (nd != 1 || bad) {
                fprintf(stderr, "%s: antenna %d file \"%s\" needs one %%d for the subband with NSUBBAND %d\n", path,
                        a, c->files[a], c->nsubband);
                return -1;
            }
        }
    return 0;
}

/* ---- streaming reader: subintegration s of every (subband, antenna) stream into one pinned set */
typedef struct {
    const conf_t* c;
    uint8_t** rows;        /* [nsubband * nant] buffers of `bytes` */
    size_t bytes;          /* bytes of one subintegration (NUMFFTS + 1 FFTs) */
    size_t stride;         /* bytes between successive subintegrations (NUMFFTS FFTs) */
    int s;                 /* subintegration to read */
    int status;            /* 0 ok, 1 error (reported) */
} read_job_t;

static void stream_name(const conf_t* c, int a, int sb, char* out, size_t n)
{
    if (c->nsubband > 1) snprintf(out, n, c->files[a], sb);
    else snprintf(out, n, "%s", c->files[a]);
}

static void* read_subint(void* arg)
{
    read_job_t* j = (read_job_t*)arg;
    const conf_t* c = j->c;
    j->status = 0;
    char name[4096];
    for (int sb = 0; sb < c->nsubband && !j->status; sb++)
        for (int a = 0; a < c->nant && !j->status; a++) {
            stream_name(c, a, sb, name, sizeof name);
            FILE* f = fopen(name, "rb");
            if (!f) {
                fprintf(stderr, "Problem with file %s - does it exist?\n", name);
                j->status = 1;
                break;
            }
            size_t got = 0;
            if (fseeko(f, (off_t)(j->stride * (size_t)j->s), SEEK_SET) == 0)
                got = fread(j->rows[sb * c->nant + a], 1, j->bytes, f);
            fclose(f);
            if (got != j->bytes) {
                fprintf(stderr, "Error: Problem reading data (Read %zu of %zu bytes from %s, subintegration %d)\n",
                        got, j->bytes, name, j->s);
                j->status = 1;
            }
        }
    return NULL;
}

/* vis: (re, im) pairs, ap: (amplitude, phase) pairs of the same visibilities (fxc_get_amp_phase) */
static void write_visout(const char* path, const float* vis, const float* ap, int nbl, int np2, int nchan, double bw)
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
                const size_t e = 2 * (((size_t)b * np2 + p) * nchan + c);
                fprintf(f, " %11.6f %11.6f", vis[e], vis[e + 1]);
                fprintf(f, " %11.6f %10.6f", ap[e], ap[e + 1]);
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
    int xmode_cli = -1, fstage_cli = -1, normalize = 1, nsubint_cli = 0;
    for (int i = 1; i < argc; i++) {
        if (!strcmp(argv[i], "-o") && i + 1 < argc) out_path = argv[++i];
        else if (!strcmp(argv[i], "-b") && i + 1 < argc) bin_path = argv[++i];
        else if (!strcmp(argv[i], "-x") && i + 1 < argc) {
            i++;
            xmode_cli = parse_xmode(argv[i]);
        } else if (!strcmp(argv[i], "-f") && i + 1 < argc) {
            i++;
            fstage_cli = parse_fstage(argv[i]);
        } else if (!strcmp(argv[i], "-s") && i + 1 < argc) nsubint_cli = atoi(argv[++i]);
        else if (!strcmp(argv[i], "-n")) normalize = 0;
        else if (argv[i][0] != '-') conf_path = argv[i];
        else {
            fprintf(stderr,
                    "usage: %s [config.conf] [-o vis.out] [-b vis.bin] [-x plain|tc|fp8] [-f fft|tc32|tc16] "
                    "[-s nsubint] [-n]\n",
                    argv[0]);
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
    cfg.xmode = xmode_cli >= 0 ? xmode_cli : c.xmode;
    cfg.fstage = fstage_cli >= 0 ? fstage_cli : c.fstage;
    cfg.nsubband = c.nsubband;
    cfg.sb_spacing = c.sbspacing;
    const int nsubint = nsubint_cli > 0 ? nsubint_cli : c.nsubint;
    const size_t bytes = fxc_subint_bytes(&cfg);
    /* bytes per NUMFFTS FFTs of one stream: the subintegration less its one-FFT slack */
    fxc_config one = cfg;
    one.numffts = 0;
    const size_t stride = bytes - fxc_subint_bytes(&one);
    const int nrow = c.nsubband * c.nant;

    /* two pinned buffer sets: the reader thread fills one while the GPU correlates the other */
    uint8_t** rows[2];
    for (int b = 0; b < 2; b++) {
        rows[b] = calloc(nrow, sizeof(uint8_t*));
        for (int r = 0; r < nrow; r++) {
            void* p = NULL;
            if (fxc_host_alloc(&p, bytes) != FXC_OK) p = malloc(bytes);
            rows[b][r] = p;
        }
    }
    read_job_t first = {&c, rows[0], bytes, stride, 0, 0};
    read_subint(&first);
    if (first.status) return 1;
    fxc_ctx* ctx = NULL;
    int st = fxc_create(&cfg, &ctx);
    if (st != FXC_OK) {
        fprintf(stderr, "fxcorr: %s (cuda error %d)\n", fxc_strerror(st), fxc_last_cuda_error());
        return 2;
    }
    const int nbl = fxc_num_baselines(&cfg);
    const size_t nvis = fxc_vis_count(&cfg);
    float* vis = NULL;
    if (fxc_host_alloc((void**)&vis, 2 * sizeof(float) * nvis) != FXC_OK) vis = malloc(2 * sizeof(float) * nvis);
    float* ap = malloc(2 * sizeof(float) * nvis);
    int* counts = malloc(sizeof(int) * (nbl + c.nant));
    double* d = malloc(3 * sizeof(double) * c.nant);
    FILE* fbin = bin_path ? fopen(bin_path, "wb") : NULL;
    if (bin_path && !fbin) {
        fprintf(stderr, "Error opening %s for writing\n", bin_path);
        return 1;
    }

    for (int s = 0; s < nsubint; s++) {
        uint8_t** cur = rows[s & 1];
        /* delay polynomial of FFT k0 + k in the subintegration's own FFT index k */
        const double k0 = (double)s * c.numffts;
        for (int a = 0; a < c.nant; a++) {
            const double q = c.delays[3 * a], l = c.delays[3 * a + 1], c0 = c.delays[3 * a + 2];
            d[3 * a] = q;
            d[3 * a + 1] = s ? l + 2.0 * q * k0 : l;
            d[3 * a + 2] = s ? c0 + l * k0 + q * k0 * k0 : c0;
        }
        /* the other buffer set was last read by the previous subintegration's copies, which
           fxc_get_visibilities waited for: the reader may overwrite it while this one runs */
        pthread_t reader;
        read_job_t next = {&c, rows[(s + 1) & 1], bytes, stride, s + 1, 0};
        int threaded = 0;
        if (s + 1 < nsubint) threaded = pthread_create(&reader, NULL, read_subint, &next) == 0;
        st = fxc_reset(ctx);
        if (st == FXC_OK) st = fxc_process_host(ctx, (const uint8_t* const*)cur, d, c.offsets, 0, c.numffts);
        if (st == FXC_OK) st = fxc_get_visibilities(ctx, vis, counts, normalize);
        if (st == FXC_OK) st = fxc_get_amp_phase(ctx, ap, normalize);
        if (threaded) pthread_join(reader, NULL);
        else if (s + 1 < nsubint) read_subint(&next);
        if (st != FXC_OK) {
            fprintf(stderr, "fxcorr: %s (cuda error %d)\n", fxc_strerror(st), fxc_last_cuda_error());
            return 2;
        }
        char base[4096], name[4200];
        if (nsubint > 1) snprintf(base, sizeof base, "%s.%d", out_path, s);
        else snprintf(base, sizeof base, "%s", out_path);
        const int np2 = c.npol * c.npol;
        for (int sb = 0; sb < c.nsubband; sb++) {
            /* one text file per subband: <out>[.<subint>][.sb<subband>] */
            if (c.nsubband > 1) snprintf(name, sizeof name, "%s.sb%d", base, sb);
            else snprintf(name, sizeof name, "%s", base);
            const size_t o = 2 * (size_t)sb * (nbl + c.nant) * np2 * c.nchan;
            write_visout(name, vis + o, ap + o, nbl, np2, c.nchan, c.bw);
        }
        if (fbin) {
            const int32_t hdr[4] = {c.nsubband, nbl + c.nant, c.npol * c.npol, c.nchan};
            fwrite(hdr, sizeof hdr, 1, fbin);
            fwrite(counts, sizeof(int), nbl + c.nant, fbin);
            fwrite(vis, 2 * sizeof(float), nvis, fbin);
        }
        if (s + 1 < nsubint && next.status) return 1;
    }
    if (fbin) fclose(fbin);
    fxc_destroy(ctx);
    return 0;
}
