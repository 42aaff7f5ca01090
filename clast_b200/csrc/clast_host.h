// clast_host.h -- the drop-in command line as a library call.
#pragma once

#ifdef __cplusplus
extern "C" {
#endif

/* Runs the reference's command line (`clast -t ... -q ... -o ...`, flags of
 * PARAMETER_GUIDE) on the GPU: truncates the -o file and appends the
 * 10-column TSV.  Returns 0 on success; otherwise a non-zero code and the
 * message in err_buf.  1 usage, 2 endless-load input, 3 I/O, 4 bad '@' line,
 * 5 no CUDA device, 6 device-path error, 7 internal. */
int clast_cli_main(int argc, const char* const* argv, char* err_buf, int err_len);

#ifdef __cplusplus
}
#endif
