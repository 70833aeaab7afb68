// Frame readers for the oracle build of the CTBB_ICD reference (test
// infrastructure only). See ctbb/ctbb_read.h for the file layout.
#include "ctbb/ctbb_read.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>

void ReadBinaryFrame(FILE* fp, int frame_idx, size_t n_channels, size_t n_rows, float* output,
                     size_t offset) {
    const size_t n = n_channels * n_rows;
    const long long pos = (long long)offset + (long long)frame_idx * (long long)(n * sizeof(float));
    if (fseeko(fp, (off_t)pos, SEEK_SET) != 0 || fread(output, sizeof(float), n, fp) != n) {
        std::fprintf(stderr, "ReadBinaryFrame: short read at frame %d\n", frame_idx);
        std::exit(1);
    }
}

static void unsupported(const char* what) {
    std::fprintf(stderr, "%s: PTR/IMA raw formats are not available in this build\n", what);
    std::exit(1);
}

float ReadPTRTubeAngle(FILE*, int, size_t, size_t) {
    unsupported("ReadPTRTubeAngle");
    return 0.0f;
}
float ReadPTRTablePosition(FILE*, int, size_t, size_t) {
    unsupported("ReadPTRTablePosition");
    return 0.0f;
}
void ReadPTRFrame(FILE*, int, size_t, size_t, float*) { unsupported("ReadPTRFrame"); }
float ReadIMATubeAngle(FILE*, int, size_t, size_t, int, size_t) {
    unsupported("ReadIMATubeAngle");
    return 0.0f;
}
float ReadIMATablePosition(FILE*, int, size_t, size_t, int, size_t) {
    unsupported("ReadIMATablePosition");
    return 0.0f;
}
void ReadIMAFrame(FILE*, int, size_t, size_t, float*, int, size_t) { unsupported("ReadIMAFrame"); }
