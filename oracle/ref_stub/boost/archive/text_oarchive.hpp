// Minimal stand-in so that the reference's parameters.h / stats.h parse without
// Boost; only the friend declaration of boost::serialization::access is used.
#pragma once
namespace boost { namespace serialization { class access {}; } }
