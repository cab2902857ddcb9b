/* A C11 program that runs the whole path through include/prr.h with no
 * Python or torch in the process: a packet file (argv[1]) is parsed,
 * decoded and developed to planar Rec.2020 on device 0 by
 * prr_decode_develop_host, from and into plain malloc'ed host memory; the
 * three f32 planes go to argv[2], the skipped tiles and max_qscale to
 * stdout. */
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
    if (argc < 3) return 2;
    size_t n = 0;
    unsigned char* pkt = read_file(argv[1], &n);
    if (!pkt) return 2;
    prr_error err;
    prr_frame_info info;
    uint8_t max_qscale = 0;
    int rc = prr_parse_frame(pkt, n, &info, &max_qscale, &err);
    if (rc != PRR_OK) {
        fprintf(stderr, "parse: %s\n", prr_status_string(rc));
        return 3;
    }
    prr_params params;
    rc = prr_params_new(&info.header, (uint32_t)info.header.quant_matrix[0] * max_qscale, &params);
    if (rc != PRR_OK) return 3;
    prr_ctx* ctx = NULL;
    rc = prr_ctx_create(0, NULL, &ctx);
    if (rc != PRR_OK) {
        fprintf(stderr, "context: %s\n", prr_status_string(rc));
        return 4;
    }
    const size_t npx = (size_t)info.header.width * info.header.height;
    float* planes = malloc(3 * npx * sizeof(float));
    uint64_t* skipped = malloc((info.ntiles ? info.ntiles : 1) * sizeof(uint64_t));
    prr_decode_result res;
    res.skipped = skipped;
    res.skipped_cap = info.ntiles;
    rc = prr_decode_develop_host(ctx, pkt, n, PRR_IDCT_APPLE, &params, PRR_STAGE_REC2020, PRR_PLANAR, planes,
                                 planes + npx, planes + 2 * npx, npx, &res, &err);
    if (rc != PRR_OK) {
        fprintf(stderr, "decode_develop: %s\n", prr_status_string(rc));
        return 5;
    }
    FILE* out = fopen(argv[2], "wb");
    if (!out || fwrite(planes, sizeof(float), 3 * npx, out) != 3 * npx) return 6;
    fclose(out);
    printf("max_qscale=%u\nskipped=", (unsigned)res.max_qscale);
    for (uint64_t i = 0; i < res.n_skipped && i < res.skipped_cap; i++) printf(i ? ",%llu" : "%llu", (unsigned long long)skipped[i]);
    printf("\n");
    prr_ctx_destroy(ctx);
    free(skipped);
    free(planes);
    free(pkt);
    return 0;
}
