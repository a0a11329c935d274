/* JPEG decoding for the image reader (hpm_io.cpp). */
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

/* out_ch 1: 8-bit gray as cv::imread(IMREAD_GRAYSCALE) returns it; 3: B, G, R
 * as IMREAD_COLOR.  HPM_OK or HPM_ERR_IO. */
int hpm_decode_jpeg(const uint8_t *data, size_t n, std::vector<uint8_t> &px, int *w, int *h, int out_ch);
/* Width and height (after the EXIF orientation) from the markers before the
 * first scan, without decoding. */
int hpm_jpeg_size(const uint8_t *data, size_t n, int *w, int *h);
