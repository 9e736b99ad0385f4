/* TEST INFRASTRUCTURE ONLY: vpl.h includes the LibImportance header (absent from the
 * reference tree) for one pointer member; a forward declaration is all it needs. */
#pragma once
namespace Renzoku { namespace Vorba { class ImportanceManager; } }
