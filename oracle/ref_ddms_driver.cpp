// C entry point over the reference's CPU restatement of the DDMS dynamic
// programming (cother-scores-optimizer/ddms.cxx:388-436, class CSO_DDMS).
// Used only by the tests to pin the oracle's DDMS against the reference's
// own code. CSO_DDMS::CalculateDDMS returns rint(16 * top-3 segment sum), or
// -777 when (len >> 2) < DSTSEGM for either list.
#include "ddms.h"

extern "C" float ref_ddms_scaled_sum(const int* list1, const int* list2)
{
    static CSO_DDMS ddms;
    return ddms.CalculateDDMS(const_cast<int*>(list1), const_cast<int*>(list2));
}
