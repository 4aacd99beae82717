// sleek_validate.cpp -- checks a compressed file against every rule the device
// decoders enforce (sleek_validate_stream), without touching a GPU.
//   sleek_validate compressed_file_name single|double
// Prints the stream's layout and "valid", or the first problem and its chunk;
// exit status 0 for a valid stream, 255 otherwise.
#include <cstdio>
#include <cstring>
#include <vector>

#include "sleek_capi.h"

int main(int argc, char* argv[])
{
  if (argc != 3 || (std::strcmp(argv[2], "single") != 0 && std::strcmp(argv[2], "double") != 0)) {
    printf("USAGE: %s compressed_file_name single|double\n\n", argv[0]);
    return -1;
  }
  FILE* const f = fopen(argv[1], "rb");
  if (!f) {
    fprintf(stderr, "ERROR: cannot read %s\n\n", argv[1]);
    return -1;
  }
  fseek(f, 0, SEEK_END);
  const long long len = ftell(f);
  fseek(f, 0, SEEK_SET);
  std::vector<unsigned char> buf(static_cast<size_t>(len > 0 ? len : 0));
  const bool ok = len <= 0 || static_cast<long long>(fread(buf.data(), 1, buf.size(), f)) == len;
  fclose(f);
  if (!ok) {
    fprintf(stderr, "ERROR: cannot read %s\n\n", argv[1]);
    return -1;
  }
  sleek_stream_info info;
  const int rc = sleek_validate_stream(buf.data(), len, argv[2][0] == 's' ? 4 : 8, &info);
  printf("file size: %lld bytes\n", len);
  printf("original size: %lld bytes\n", info.insize);
  printf("chunks: %lld (%lld stored raw)\n", info.chunks, info.raw_chunks);
  printf("stream bytes checked: %lld\n", info.stream_bytes);
  if (rc == SLEEK_OK) {
    printf("valid\n");
    return 0;
  }
  printf("INVALID: %s", sleek_stream_reason_string(info.reason));
  if (info.bad_chunk >= 0) printf(" at chunk %lld", info.bad_chunk);
  printf("\n");
  return -1;
}
