// Plumbing shim for BOOST_CURRENT_FUNCTION (used only in THROW messages).
#pragma once
#define BOOST_CURRENT_FUNCTION __PRETTY_FUNCTION__
