/// @file properties.h
/// @brief Key/value parameter set (interface of FastLBP's include/lbp/properties.h:21-59).
/// getStringAs<T>() requires the stored value to have exactly type T; on a
/// mismatch it prints "get properties error" and returns T().
#pragma once

#include <any>
#include <iostream>
#include <map>
#include <string>

namespace lbp {

typedef std::string PropertyKey;
typedef std::any PropertyValue;

class PropertySet : private std::map<PropertyKey, PropertyValue> {
public:
    PropertySet() = default;
    ~PropertySet() = default;

    PropertySet &set(const PropertyKey &key, const PropertyValue &val) {
        (*this)[key] = val;
        return *this;
    }

    const PropertyValue &get(const PropertyKey &key) const {
        auto x = find(key);
        if (x == end()) {
            std::cerr << "Did not find key: " << key << std::endl;
            static const PropertyValue empty;
            return empty;
        }
        return x->second;
    }

    template <typename ValueType>
    ValueType getStringAs(const PropertyKey &key) const {
        const PropertyValue &val = get(key);
        if (val.type() == typeid(ValueType)) return std::any_cast<ValueType>(val);
        std::cerr << "get properties error" << std::endl;
        return ValueType();
    }

    bool hasKey(const PropertyKey &key) const { return find(key) != end(); }
};

}  // namespace lbp
