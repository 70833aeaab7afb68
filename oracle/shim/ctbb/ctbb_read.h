// Declarations of the raw-frame reader functions that the CTBB_ICD reference
// calls from setup.cpp:288, 307-310, 322-324. The real ctbb_read / fct_read
// library is not public; this header and oracle/shim/ctbb_read.cpp stand in
// for it in the oracle build (test infrastructure only).
//
// Only the FileType 0 (flat binary) reader has a body: frame `frame_idx` is
// n_channels*n_rows float32 values at byte offset
// offset + frame_idx*n_channels*n_rows*4, channel-major with the row index
// fastest (the layout load_raw's transpose at setup.cpp:291-298 expects).
// The synthetic phantom generator writes files in exactly this layout.
#pragma once

#include <cstddef>
#include <cstdio>

void ReadBinaryFrame(FILE* fp, int frame_idx, size_t n_channels, size_t n_rows, float* output,
                     size_t offset);

float ReadPTRTubeAngle(FILE* fp, int frame_idx, size_t n_channels, size_t n_rows);
float ReadPTRTablePosition(FILE* fp, int frame_idx, size_t n_channels, size_t n_rows);
void ReadPTRFrame(FILE* fp, int frame_idx, size_t n_channels, size_t n_rows, float* output);

float ReadIMATubeAngle(FILE* fp, int frame_idx, size_t n_channels, size_t n_rows, int subtype,
                       size_t offset);
float ReadIMATablePosition(FILE* fp, int frame_idx, size_t n_channels, size_t n_rows, int subtype,
                           size_t offset);
void ReadIMAFrame(FILE* fp, int frame_idx, size_t n_channels, size_t n_rows, float* output,
                  int subtype, size_t offset);
