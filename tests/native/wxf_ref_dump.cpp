// Test infrastructure, compiled only where the reference tree is present: decodes a WXF file with
// the reference's own parser (wxf/wxf.cpp) and prints it as canonical text -- integers, "strings",
// [lists], <|key->value, ...|> -- so the CPU tests can compare it with the Python decoder.
#include <cstdio>
#include <fstream>
#include <iterator>
#include <string>
#include <vector>

#include "wxf.hpp"

using hg::wxf::Parser;

static void dump(Parser& p, std::string& out) {
    const uint8_t tok = p.data()[p.position()];
    switch (tok) {
        case 'C': out += std::to_string(p.read_int8()); break;
        case 'j': out += std::to_string(p.read_int16()); break;
        case 'i': out += std::to_string(p.read_int32()); break;
        case 'L': out += std::to_string(p.read_int64()); break;
        case 'S': out += "\"" + p.read_string() + "\""; break;
        case 's': out += p.read_symbol(); break;
        case 'f':
            p.read_function([&](const std::string& head, size_t n, Parser& q) {
                out += head == "List" ? "[" : head + "[";
                for (size_t i = 0; i < n; ++i) {
                    if (i) out += ",";
                    dump(q, out);
                }
                out += "]";
            });
            break;
        case 'A': {
            out += "<|";
            bool first = true;
            p.read_association_generic([&](Parser& k, Parser& v) {
                if (!first) out += ",";
                first = false;
                dump(k, out);
                out += "->";
                dump(v, out);
            });
            out += "|>";
            break;
        }
        default: out += "?"; p.skip_value(); break;
    }
}

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    std::ifstream f(argv[1], std::ios::binary);
    std::vector<uint8_t> bytes((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    Parser p(bytes);
    p.skip_header();
    std::string out;
    dump(p, out);
    std::printf("%s\n", out.c_str());
    return p.at_end() ? 0 : 1;
}
