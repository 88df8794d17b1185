/*
 * Status codes returned by every entry point of the FFT C ABI.
 *
 * The numeric values are part of the drop-in contract: callers written
 * against hicann/sip compare against these constants.  They follow
 * core/utils/include/utils/aspb_status.h:14-25 of the reference.
 */
#ifndef SIP_B200_ASPB_STATUS_H
#define SIP_B200_ASPB_STATUS_H

#include <cstdint>

namespace AsdSip {
using AspbStatus = int32_t;

enum ErrorType : int {
    ACL_SUCCESS = 0,
    ACL_ERROR_INVALID_PARAM = 100000,
    ACL_ERROR_OP_INPUT_NOT_MATCH = 100021,
    ACL_ERROR_OP_OUTPUT_NOT_MATCH = 100022,
    ACL_ERROR_UNSUPPORTED_DATA_TYPE = 100026,
    ACL_ERROR_FORMAT_NOT_MATCH = 100027,
    ACL_ERROR_API_NOT_SUPPORT = 200001,
    ACL_ERROR_INTERNAL_ERROR = 500000
};
}  // namespace AsdSip

#endif
