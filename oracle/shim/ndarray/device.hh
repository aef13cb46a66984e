// Empty stand-in for hguo/ndarray's device header (the oracle build has no GPU).
// TEST INFRASTRUCTURE ONLY.
#pragma once
