// ffb_flame_xml.hpp -- `.flame` XML import (ffb_flame_xml.cpp).
#pragma once

#include <string>
#include <vector>

namespace ffb {

// Every <flame> / <jwf-flame> of the document as a `.fae` config (JSON
// text), in document order.  Throws std::runtime_error with the reason.
std::vector<std::string> flame_xml_import(const std::string& xml);

}  // namespace ffb
