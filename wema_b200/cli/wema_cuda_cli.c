/*
 * wema_cuda_cli.c - the reference CLI's command line (main.c:18-218, 223-490)
 * on top of libwema_cuda.
 *
 * Flags, defaults, checks and messages follow main.c's parse_args: -i/-o,
 * -a, --fl, --fh (clamped to fps/2 - 1e-4 once the rate is known, main.c:248),
 * --temporal-window (4..256), --no-edge-aware, --bilateral-filter, --color,
 * --haar, --batch (1..256), --threads, -v, -h.  Routing follows main.c:355:
 * IIR luma with a batch size above 1 takes the reference's batch route (its
 * threshold form, the guided filter always on); everything else the
 * single-frame route.
 *
 * Frames are raw RGB24 ("rawvideo rgb24", what the reference's FFmpeg pipes
 * carry, ffmpeg_io.c:264-323): no decoder or encoder is on this path, so the
 * size and rate that ffprobe would report come from --size WxH and --fps.
 * "-" reads stdin / writes stdout.  The default output is <input>.wema.rgb
 * (main.c:50-61 appends .wema.mkv).  --ff-codec / --ff-option are accepted
 * and ignored (no encoder).  A partial frame at the end of the input is an
 * error, as in ffio_read_frame (ffmpeg_io.c:277-280).
 */
#define _POSIX_C_SOURCE 200809L
#include <stdbool.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "wema_cuda.h"

#define WINDOW_DEF 32
#define WINDOW_MAX 256
#define BATCH_DEF 64
#define BATCH_MAX 256

typedef struct {
    const char *input_path, *output_path, *ff_codec, *ff_options;
    float amp_factor, f_low, f_high, fps;
    int temporal_window, batch_size, num_threads, width, height;
    bool verbose, edge_aware, bilateral_temp, color_mode, use_iir;
} CliConfig;

static void print_usage(const char *prog) {
    fprintf(stderr,
            "Usage: %s -i <input> --size <W>x<H> --fps <rate> [-o <output>] [options]\n"
            "\n"
            "Options:\n"
            "  -i, --input <file>     Input raw RGB24 frames ('-' = stdin) (required)\n"
            "  -o, --output <file>    Output raw RGB24 frames (default: input.wema.rgb, '-' = stdout)\n"
            "  --size <W>x<H>         Frame size (required: raw frames carry none)\n"
            "  --fps <rate>           Frame rate in Hz (required)\n"
            "  -a, --amp <factor>     Amplification factor (default: 120)\n"
            "  --fl <freq>            Low frequency cutoff in Hz (default: 0.5)\n"
            "  --fh <freq>            High frequency cutoff in Hz (default/max: half of framerate)\n"
            "  --ff-codec <codec>     Accepted for compatibility; ignored (no encoder)\n"
            "  --ff-option <opts>     Accepted for compatibility; ignored\n"
            "  --temporal-window <n>  Temporal window size (default: 32, min:4, max: 256)\n"
            "  --no-edge-aware        Disable edge-aware guided filter\n"
            "  --bilateral-filter     Enable bilateral temporal filtering\n"
            "  --color                Enable color mode (amplify color channels)\n"
            "  --haar                 Sliding-window temporal filter instead of IIR\n"
            "  --batch <n>            Batch size (default: 64; > 1 selects the batch route)\n"
            "  --threads <n>          Number of threads (accepted; the GPU does the work)\n"
            "  -v, --verbose          Verbose output\n"
            "  -h, --help             Show this help\n",
            prog);
}

static int need(int i, int argc, const char *flag) {
    if (i >= argc) {
        fprintf(stderr, "Error: %s requires an argument\n", flag);
        return -1;
    }
    return 0;
}

/* 0: run; 1: help printed; -1: error (message printed) */
static int parse_args(int argc, char **argv, CliConfig *c) {
    memset(c, 0, sizeof *c);
    c->amp_factor = 120.0f;
    c->f_low = 0.5f;
    c->f_high = 1048576.0f;
    c->temporal_window = WINDOW_DEF;
    c->edge_aware = true;
    c->use_iir = true;
    c->batch_size = BATCH_DEF;
    for (int i = 1; i < argc; i++) {
        const char *a = argv[i];
        if (!strcmp(a, "-i") || !strcmp(a, "--input")) {
            if (need(++i, argc, "-i")) return -1;
            c->input_path = argv[i];
        } else if (!strcmp(a, "-o") || !strcmp(a, "--output")) {
            if (need(++i, argc, "-o")) return -1;
            c->output_path = argv[i];
        } else if (!strcmp(a, "--size")) {
            if (need(++i, argc, "--size")) return -1;
            if (sscanf(argv[i], "%dx%d", &c->width, &c->height) != 2 || c->width < 1 || c->height < 1) {
                fprintf(stderr, "Error: --size takes <W>x<H> with positive sizes\n");
                return -1;
            }
        } else if (!strcmp(a, "--fps")) {
            if (need(++i, argc, "--fps")) return -1;
            c->fps = strtof(argv[i], NULL);
            if (!(c->fps > 0)) {
                fprintf(stderr, "Error: frame rate must be positive\n");
                return -1;
            }
        } else if (!strcmp(a, "-a") || !strcmp(a, "--amp")) {
            if (need(++i, argc, "-a")) return -1;
            c->amp_factor = strtof(argv[i], NULL);
            if (c->amp_factor <= 0) {
                fprintf(stderr, "Error: amplification factor must be positive\n");
                return -1;
            }
        } else if (!strcmp(a, "--fl")) {
            if (need(++i, argc, "--fl")) return -1;
            c->f_low = strtof(argv[i], NULL);
            if (c->f_low < 0) {
                fprintf(stderr, "Error: low frequency must be non-negative\n");
                return -1;
            }
        } else if (!strcmp(a, "--fh")) {
            if (need(++i, argc, "--fh")) return -1;
            c->f_high = strtof(argv[i], NULL);
            if (c->f_high <= 0) {
                fprintf(stderr, "Error: high frequency must be positive\n");
                return -1;
            }
        } else if (!strcmp(a, "--temporal-window")) {
            if (need(++i, argc, "--temporal-window")) return -1;
            c->temporal_window = atoi(argv[i]);
            if (c->temporal_window < 4) {
                fprintf(stderr, "Error: temporal window must be at least 4\n");
                return -1;
            }
            if (c->temporal_window > WINDOW_MAX) {
                fprintf(stderr, "Error: temporal window cannot exceed %d\n", WINDOW_MAX);
                return -1;
            }
        } else if (!strcmp(a, "--ff-codec")) {
            if (need(++i, argc, "--ff-codec")) return -1;
            c->ff_codec = argv[i];
        } else if (!strcmp(a, "--ff-option")) {
            if (need(++i, argc, "--ff-option")) return -1;
            c->ff_options = argv[i];
        } else if (!strcmp(a, "-v") || !strcmp(a, "--verbose")) {
            c->verbose = true;
        } else if (!strcmp(a, "--no-edge-aware")) {
            c->edge_aware = false;
        } else if (!strcmp(a, "--bilateral-filter")) {
            c->bilateral_temp = true;
        } else if (!strcmp(a, "--color")) {
            c->color_mode = true;
        } else if (!strcmp(a, "--haar")) {
            c->use_iir = false;
        } else if (!strcmp(a, "--batch")) {
            if (need(++i, argc, "--batch")) return -1;
            c->batch_size = atoi(argv[i]);
            if (c->batch_size < 1) {
                fprintf(stderr, "Error: batch size must be at least 1\n");
                return -1;
            }
            if (c->batch_size > BATCH_MAX) {
                fprintf(stderr, "Error: batch size cannot exceed %d\n", BATCH_MAX);
                return -1;
            }
        } else if (!strcmp(a, "--threads")) {
            if (need(++i, argc, "--threads")) return -1;
            c->num_threads = atoi(argv[i]);
            if (c->num_threads < 0) {
                fprintf(stderr, "Error: thread count must be non-negative\n");
                return -1;
            }
        } else if (!strcmp(a, "-h") || !strcmp(a, "--help")) {
            print_usage(argv[0]);
            return 1;
        } else {
            fprintf(stderr, "Error: Unknown option: %s\n", a);
            return -1;
        }
    }
    if (!c->input_path) {
        fprintf(stderr, "Error: Input file required (-i)\n");
        return -1;
    }
    if (c->f_low >= c->f_high) {
        fprintf(stderr, "Error: Low frequency must be less than high frequency\n");
        return -1;
    }
    if (c->width < 1 || c->fps <= 0) {
        fprintf(stderr, "Error: raw RGB24 input needs --size <W>x<H> and --fps <rate>\n");
        return -1;
    }
    return 0;
}

/* bytes read into buf (< n only at the end of the input) */
static size_t read_full(FILE *f, unsigned char *buf, size_t n) {
    size_t got = 0;
    while (got < n) {
        size_t r = fread(buf + got, 1, n - got, f);
        if (r == 0) break;
        got += r;
    }
    return got;
}

int main(int argc, char **argv) {
    CliConfig c;
    int rc = parse_args(argc, argv, &c);
    if (rc == 1) return 0;
    if (rc < 0) {
        print_usage(argv[0]);
        return 1;
    }
    if (c.f_high > c.fps / 2.0f - 0.0001f) c.f_high = c.fps / 2.0f - 0.0001f;   /* main.c:248 */
    if (c.f_low >= c.f_high) {
        fprintf(stderr, "Error: Low frequency must be less than high frequency\n");
        return 1;
    }
    char *auto_out = NULL;
    if (!c.output_path) {
        size_t len = strlen(c.input_path);
        const char *dot = strrchr(c.input_path, '.');
        const char *slash = strrchr(c.input_path, '/');
        size_t base = (dot && (!slash || dot > slash)) ? (size_t)(dot - c.input_path) : len;
        auto_out = malloc(base + 16);
        if (!auto_out) {
            fprintf(stderr, "Error: Failed to allocate output path\n");
            return 1;
        }
        memcpy(auto_out, c.input_path, base);
        strcpy(auto_out + base, ".wema.rgb");
        c.output_path = auto_out;
    }
    const bool batch_route = c.use_iir && c.batch_size > 1 && !c.color_mode;   /* main.c:355 */
    if (c.ff_codec || c.ff_options)
        fprintf(stderr, "Note: --ff-codec / --ff-option ignored (raw RGB24 output)\n");
    if (c.verbose) {
        fprintf(stderr, "Input: %s\n  Size: %dx%d\n  FPS: %.3f\nOutput: %s\nSettings:\n", c.input_path,
                c.width, c.height, c.fps, c.output_path);
        fprintf(stderr, "  Amplification: %.1f\n", c.amp_factor);
        fprintf(stderr, "  Frequency band: %.2f - %.2f Hz\n", c.f_low, c.f_high);
        fprintf(stderr, "  Temporal window: %d frames\n", c.temporal_window);
        fprintf(stderr, "  Temporal filter: %s\n", c.use_iir ? "IIR (fast)" : "Haar wavelet");
        fprintf(stderr, "  Bilateral temporal: %s\n", c.bilateral_temp ? "enabled" : "disabled");
        fprintf(stderr, "  Edge-aware filter: %s\n", (c.edge_aware || batch_route) ? "enabled" : "disabled");
        fprintf(stderr, "  Color mode: %s\n", c.color_mode ? "enabled" : "disabled");
        if (c.use_iir) fprintf(stderr, "  Batch size: %d frames (%s route)\n", c.batch_size,
                               batch_route ? "batch" : "single-frame");
    }

    wema_cuda_config cfg;
    wema_cuda_config_default(&cfg, c.width, c.height, c.fps);
    cfg.amp_factor = c.amp_factor;
    cfg.f_low = c.f_low;
    cfg.f_high = c.f_high;
    cfg.temporal_window = c.temporal_window;
    cfg.edge_aware = batch_route ? 1 : c.edge_aware;      /* the batch route always filters */
    cfg.bilateral_temp = c.bilateral_temp;
    cfg.color_mode = c.color_mode;
    cfg.use_iir = c.use_iir;
    cfg.threshold_form = batch_route ? WEMA_CUDA_THR_BATCH : WEMA_CUDA_THR_SINGLE;

    FILE *in = strcmp(c.input_path, "-") ? fopen(c.input_path, "rb") : stdin;
    if (!in) {
        fprintf(stderr, "Error: Cannot open input: %s\n", c.input_path);
        free(auto_out);
        return 1;
    }
    FILE *out = strcmp(c.output_path, "-") ? fopen(c.output_path, "wb") : stdout;
    if (!out) {
        fprintf(stderr, "Error: Cannot open output: %s\n", c.output_path);
        if (in != stdin) fclose(in);
        free(auto_out);
        return 1;
    }
    wema_cuda_session *s = NULL;
    if (wema_cuda_session_create(&cfg, &s) != 0) {
        fprintf(stderr, "Error: Failed to initialize WEMA: %s\n", wema_cuda_last_error());
        if (in != stdin) fclose(in);
        if (out != stdout) fclose(out);
        free(auto_out);
        return 1;
    }
    const size_t fb = (size_t)c.width * c.height * 3;
    unsigned char *fin = malloc(fb), *fout = malloc(fb);
    long frames = 0;
    int status = 0;
    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    while (fin && fout) {
        const size_t got = read_full(in, fin, fb);
        if (got == 0) break;
        if (got < fb) {
            fprintf(stderr, "Error: partial frame at the end of the input (%zu of %zu bytes)\n", got, fb);
            status = 1;
            break;
        }
        if (wema_cuda_process_host_u8(s, fin, fout) != 0) {
            fprintf(stderr, "Error: frame %ld: %s\n", frames, wema_cuda_last_error());
            status = 1;
            break;
        }
        if (fwrite(fout, 1, fb, out) != fb) {
            fprintf(stderr, "Error: write failed at frame %ld\n", frames);
            status = 1;
            break;
        }
        frames++;
        if (c.verbose && frames % 100 == 0) fprintf(stderr, "  Frame %ld\n", frames);
    }
    if (!fin || !fout) {
        fprintf(stderr, "Error: out of host memory\n");
        status = 1;
    }
    clock_gettime(CLOCK_MONOTONIC, &t1);
    if (c.verbose) {
        const double sec = (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
        fprintf(stderr, "Processed %ld frames in %.3f s (%.1f fps)\n", frames, sec,
                sec > 0 ? (double)frames / sec : 0.0);
    }
    wema_cuda_session_destroy(s);
    free(fin);
    free(fout);
    if (in != stdin) fclose(in);
    if (out != stdout) fclose(out);
    free(auto_out);
    return status;
}
