// Parser harness for the sanitizer test (tests/test_parser_fuzz.py): reads
// length-prefixed codestreams (uint32 little-endian length, then the bytes)
// from stdin and runs the header reader and the full parser on each.  Built
// with -fsanitize=address,undefined, so an out-of-bounds access or undefined
// behaviour on malformed input ends the run with a report.
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "j2k_host.h"

int main()
{
    uint32_t n;
    size_t count = 0, parsed = 0;
    while (fread(&n, 4, 1, stdin) == 1) {
        std::vector<uint8_t> b(n);
        if (n && fread(b.data(), 1, n, stdin) != n) return 2;
        tc::Parsed p;
        std::string err;
        tc_image_info info;
        tc::read_header(b.data(), b.size(), info, err);
        if (tc::parse_codestream(b.data(), b.size(), p, err) == 0) parsed++;
        count++;
    }
    printf("parsed %zu of %zu\n", parsed, count);
    return 0;
}
