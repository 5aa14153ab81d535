// Driver (ours) around the reference's own description formatters,
// FormatDescription and FormatDescriptionJSON (src/liblib/fmtdescription.h,
// header-only), compiled from where they lie by `make -C oracle fmtref` into
// _ref/libfmtref.so. Test infrastructure: it produces the golden vectors of
// tests/golden/fmt_desc_ref.json; the product never links it.
#include <cstring>
#include "fmtdescription.h"

extern "C" {

// out must hold maxoutlen + indent * (maxoutlen / 2) + 8 bytes; returns the
// number of bytes written
int ref_format_description(const char* desc, int maxoutlen, int indent, int width, int outpos, int linepos,
                           char addsep, char* out)
{
    char* p = out;
    FormatDescription(p, desc, maxoutlen, indent, width, outpos, linepos, addsep);
    return (int)(p - out);
}

int ref_format_description_json(const char* desc, int maxoutlen, int outpos, char* out)
{
    char* p = out;
    FormatDescriptionJSON(p, desc, maxoutlen, outpos);
    return (int)(p - out);
}
}
