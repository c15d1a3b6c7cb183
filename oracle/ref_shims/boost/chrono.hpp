// Plumbing shim: empty.
#pragma once
