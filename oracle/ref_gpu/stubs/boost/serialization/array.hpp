// Stand-in for the one Boost header the reference's tensor/vector.hpp
// includes: vector<> only befriends boost::serialization::access for its
// (never instantiated here) serialize() template, so a declaration suffices.
#pragma once
namespace boost
{
namespace serialization
{
class access;
}
}  // namespace boost
