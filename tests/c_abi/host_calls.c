/* A C11 consumer of include/prr.h: the host-side entry points a caller with
 * no GPU at hand can use (header and frame parsing, demosaic parameters,
 * the output matrix, status strings, the DNG container's number formats),
 * called on the packet file given as argv[1]. Prints key=value lines for the
 * test that runs it to compare with the Python mirror of the same calls. */
#include <stdio.h>
#include <stdlib.h>

#include "prr.h"

static unsigned char* read_file(const char* path, size_t* n) {
    FILE* f = fopen(path, "rb");
    if (!f) return NULL;
    fseek(f, 0, SEEK_END);
    const long size = ftell(f);
    fseek(f, 0, SEEK_SET);
    unsigned char* buf = malloc(size > 0 ? (size_t)size : 1);
    *n = buf ? fread(buf, 1, (size_t)size, f) : 0;
    fclose(f);
    return buf;
}

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    size_t n = 0;
    unsigned char* pkt = read_file(argv[1], &n);
    if (!pkt) return 2;
    prr_error err;
    size_t hlen = 0;
    const int hrc = prr_header_len(pkt, n, &hlen, &err);
    printf("header_len_rc=%d\nheader_len=%zu\n", hrc, hlen);

    prr_frame_info info;
    uint8_t max_qscale = 0;
    const int rc = prr_parse_frame(pkt, n, &info, &max_qscale, &err);
    printf("parse_frame_rc=%d\nwidth=%u\nheight=%u\ncoded_width=%u\ncoded_height=%u\n", rc,
           (unsigned)info.header.width, (unsigned)info.header.height, info.coded_width, info.coded_height);
    printf("ntiles=%u\ntiles_per_row=%u\ntile_rows=%u\nbayer=%u\nwhite=%u\nmax_qscale=%u\n", info.ntiles,
           info.tiles_per_row, info.tile_rows, (unsigned)info.header.bayer_pattern,
           (unsigned)info.header.white_level, (unsigned)max_qscale);

    prr_params p;
    const uint32_t quantizer = (uint32_t)info.header.quant_matrix[0] * max_qscale;
    const int prc = prr_params_new(&info.header, quantizer, &p);
    printf("params_rc=%d\n", prc);
    printf("cfa_phase=%d\nblack=%d\none_over_range=%.9g\nnoise=%.9g,%.9g,%.9g\nclip=%.9g,%.9g\nwb=%.9g,%.9g\n",
           p.cfa_phase, p.black, p.one_over_range, p.noise[0], p.noise[1], p.noise[2], p.clip[0], p.clip[1],
           p.wb[0], p.wb[1]);
    float m[9];
    const int mrc = prr_output_matrix(&info.header, 0, m);
    printf("matrix_rc=%d\nmatrix=", mrc);
    for (int i = 0; i < 9; i++) printf(i ? ",%.9g" : "%.9g", m[i]);
    printf("\n");

    /* A packet cut inside its header: the error's fields. */
    const int trc = prr_parse_header(pkt, 10, &info.header, &err);
    printf("truncated_rc=%d\ntruncated_code=%d\nstatus=%s\n", trc, err.code, prr_status_string(trc));

    int32_t num = 0, den = 0;
    uint32_t unum = 0, uden = 0;
    char when[20];
    const int src = prr_dng_srational(-0.3125, &num, &den);
    printf("srational_rc=%d\nsrational=%d/%d\n", src, num, den);
    const int rrc = prr_dng_rational(2.2, &unum, &uden);
    printf("rational_rc=%d\nrational=%u/%u\n", rrc, unum, uden);
    const int drc = prr_dng_date_time(3000000000ull, when);
    printf("date_rc=%d\ndate=%.19s\n", drc, when);
    printf("padded_100=%zu\nlj92_bound_256=%llu\n", prr_padded_packet_bytes(100),
           (unsigned long long)prr_lj92_tile_bound(256));
    free(pkt);
    return 0;
}
