/* Stand-in for spdlog (a network-fetched dependency of the reference, absent here) with the five
   logging calls the reference's logger/Logger.h macros expand to, so that the reference's headers
   parse in the adapter compile test. Test infrastructure only. */
#pragma once
namespace spdlog
{
template <class... A> void trace(A &&...) {}
template <class... A> void debug(A &&...) {}
template <class... A> void info(A &&...) {}
template <class... A> void warn(A &&...) {}
template <class... A> void critical(A &&...) {}
} // namespace spdlog
