// A fixed association written with the library's WXF writer (include/hgx/wxf.hpp) to argv[1]:
// integers at every width boundary, strings, nested lists, an integer-keyed association and a
// boolean. The CPU tests decode it with the Python decoder and, where the reference tree is
// present, with the reference's own WXF parser.
#include <fstream>

#include "hgx/wxf.hpp"

int main(int argc, char** argv) {
    hgx::wxf::Writer w;
    w.association(5);
    w.key("Ints");
    const int64_t ints[] = {0, 1, -1, 127, -128, 128, -129, 32767, -32768, 32768, -32769,
                            2147483647LL, -2147483648LL, 2147483648LL, -2147483649LL,
                            9223372036854775807LL, -9223372036854775807LL - 1};
    w.list(sizeof(ints) / sizeof(ints[0]));
    for (int64_t x : ints) w.integer(x);
    w.key("Text");
    w.string("multiway \xce\xbb step");
    w.key("Nested");
    w.list(2);
    w.list(0);
    w.list(3);
    w.integer(1);
    w.string("two");
    w.list(1);
    w.integer(3);
    w.key("ByState");
    w.association(2);
    w.int_key(300);
    w.association(1);
    w.key("IsInitial");
    w.boolean(true);
    w.int_key(-7);
    w.string("x");
    w.key("Flag");
    w.boolean(false);
    const auto& d = w.data();
    std::ofstream(argc > 1 ? argv[1] : "sample.wxf", std::ios::binary)
        .write(reinterpret_cast<const char*>(d.data()), static_cast<std::streamsize>(d.size()));
    return 0;
}
